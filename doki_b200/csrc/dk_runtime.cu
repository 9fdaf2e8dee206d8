/*
 * C-ABI implementation of the B200 state-vector engine (host side).
 *
 * Registers are immutable values.  A register is (buffer, pending gates):
 * registry_apply only appends a gate to a persistent, shared op list, so it
 * costs O(1) host time.  The queued gates are executed when the register is
 * read (get / prob / measure / join / density): the planner (dk_plan.c) fuses
 * them into multi-gate sweeps, which run in place when no other register
 * shares the buffer and out of place (first sweep reads the shared buffer,
 * writes a fresh one) otherwise.  Because logical amplitudes are amp / norm
 * and every sweep recomputes the norm, the result equals the reference's
 * gate-by-gate renormalised evolution (qops.c:176-261) for any grouping.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <mutex>
#include <new>
#include <vector>

#include "dk_internal.h"
#include "dk_kernels.h"

namespace {

/* A slot: one CUDA stream with its own scratch and lock.  Every
 * register belongs to the slot that created it (derived registers inherit
 * it); work on a register is queued on its slot's stream under its slot's
 * lock, so registers of different slots run concurrently on the device and a
 * thread waiting for its results does not block other slots. */
struct Slot {
	cudaStream_t st = nullptr;
	dk::Scratch scratch{};
	std::recursive_mutex mu;
};

constexpr int kMaxSlots = 64;

struct Ctx {
	std::atomic<int> inited{ 0 };
	int device = 0;
	int num_sms = 148;
	std::mutex init_mu;
	std::mutex slots_mu;
	Slot *slots[kMaxSlots] = { nullptr };
	std::atomic<int> nslots{ 0 };
	std::atomic<size_t> allocated{ 0 };
	size_t budget = 0; /* 0 = unlimited */
	int fuse = 1;
	int tile_bits = 0; /* 0: planner default */
	int fold = 0; /* pass-folding cost: 0 planner default, < 0 off */
	int tensor = 0; /* tensor-core sweeps: 0 planner default (on), < 0 off */
	int low_bits = -1; /* qubits always in a sweep's tile: < 0 planner default */
	std::atomic<unsigned long long> sweeps{ 0 }, gates{ 0 }, h2d{ 0 }, d2h{ 0 };
	/* tensor sweeps: sum of matrix entries x register amplitudes */
	std::atomic<unsigned long long> mma_entry_amps{ 0 };
	char err[256] = { 0 };
};

Ctx g;

/* slot new registers of this thread are created on */
thread_local int t_slot = 0;
/* slot of the operation in progress on this thread (set by SlotLock) */
thread_local Slot *t_active = nullptr;
#define CUR (*t_active)

/* Locks a slot for the current scope and makes it the active one. */
struct SlotLock {
	Slot *prev;
	Slot *sl;
	explicit SlotLock(int id)
	{
		prev = t_active;
		if (id < 0 || id >= kMaxSlots || !g.slots[id])
			id = 0;
		sl = g.slots[id];
		if (sl) {
			sl->mu.lock();
			t_active = sl;
		}
	}
	~SlotLock()
	{
		if (sl)
			sl->mu.unlock();
		t_active = prev;
	}
};

int create_slot(int id)
{
	Slot *sl = new (std::nothrow) Slot();
	if (!sl)
		return DK_ERR_ALLOC;
	cudaError_t e = cudaStreamCreateWithFlags(&sl->st, cudaStreamNonBlocking);
	if (e == cudaSuccess)
		e = cudaMalloc(&sl->scratch.partials,
			       sizeof(double) * dk::kMaxBlocks * dk::kPartialStride);
	if (e == cudaSuccess)
		e = cudaMalloc(&sl->scratch.u64, 4 * sizeof(unsigned long long));
	if (e == cudaSuccess)
		e = cudaMalloc(&sl->scratch.marg, 64 * sizeof(double));
	if (e != cudaSuccess) {
		snprintf(g.err, sizeof(g.err), "%s", cudaGetErrorString(e));
		cudaGetLastError();
		delete sl;
		return DK_ERR_CUDA;
	}
	g.slots[id] = sl;
	return DK_OK;
}

int cuda_fail(cudaError_t e)
{
	snprintf(g.err, sizeof(g.err), "%s", cudaGetErrorString(e));
	cudaGetLastError(); /* clear non-sticky errors */
	return e == cudaErrorMemoryAllocation ? DK_ERR_ALLOC : DK_ERR_CUDA;
}

#define CK(call)                                   \
	do {                                       \
		cudaError_t e_ = (call);           \
		if (e_ != cudaSuccess)             \
			return cuda_fail(e_);      \
	} while (0)

int ensure_init()
{
	if (g.inited.load())
		return DK_OK;
	return dk_init(-1);
}

size_t amp_bytes(int prec) { return prec == DK_C64 ? 8 : 16; }

int dev_alloc(void **p, size_t bytes)
{
	if (g.budget && g.allocated.load() + bytes > g.budget)
		return DK_ERR_BUDGET;
	cudaError_t e = cudaMallocAsync(p, bytes ? bytes : 16, CUR.st);
	if (e != cudaSuccess)
		return cuda_fail(e);
	g.allocated += bytes;
	return DK_OK;
}

void dev_free(void *p, size_t bytes)
{
	if (!p)
		return;
	cudaFreeAsync(p, CUR.st);
	g.allocated -= bytes;
}

/* ---- buffers ------------------------------------------------------------ */

void buf_release(dk_buf *b);

int buf_new(unsigned n, int prec, dk_buf **out)
{
	dk_buf *b = (dk_buf *)calloc(1, sizeof(dk_buf));
	if (!b)
		return DK_ERR_ALLOC;
	b->refcount = 1;
	b->n = n;
	b->prec = prec;
	b->bytes = amp_bytes(prec) << n;
	int rc = dev_alloc(&b->d, b->bytes);
	if (rc) {
		free(b);
		return rc;
	}
	rc = dev_alloc((void **)&b->sc, sizeof(dk_scal));
	if (rc) {
		dev_free(b->d, b->bytes);
		free(b);
		return rc;
	}
	/* pool memory is recycled: start every scalar block from zero */
	cudaError_t e = cudaMemsetAsync(b->sc, 0, sizeof(dk_scal), CUR.st);
	if (e != cudaSuccess) {
		buf_release(b);
		return cuda_fail(e);
	}
	*out = b;
	return DK_OK;
}

void buf_release(dk_buf *b)
{
	if (!b)
		return;
	if (--b->refcount > 0)
		return;
	dev_free(b->d, b->bytes);
	dev_free(b->sc, sizeof(dk_scal));
	free(b);
}

/* ---- pending op chains ------------------------------------------------- */

void gate_retain(dk_gate *gt) { __atomic_fetch_add(&gt->refcount, 1, __ATOMIC_RELAXED); }

void op_release(dk_op *op)
{
	while (op && --op->refcount == 0) {
		dk_op *prev = op->prev;
		dk_gate_free(op->gate);
		free(op);
		op = prev;
	}
}

/* ---- states ------------------------------------------------------------- */

dk_state *state_alloc(unsigned n, int prec, int slot)
{
	dk_state *s = (dk_state *)calloc(1, sizeof(dk_state));
	if (!s)
		return nullptr;
	s->n = n;
	s->prec = prec;
	s->slot = slot;
	return s;
}

void state_drop_caches(dk_state *s)
{
	free(s->marg);
	s->marg = nullptr;
	s->have_marg = 0;
	free(s->hcache);
	s->hcache = nullptr;
	s->have_phase = 0;
	s->have_norm = 0;
}

int check_live(dk_state *s)
{
	if (!s)
		return DK_ERR_ARG;
	if (s->released)
		return DK_ERR_DEAD;
	return DK_OK;
}

/* Execute the pending gates of `s` (see the file comment). */
static int flush_queued(dk_state *s);

/* Run the register's queued gates; host allocation failures (std::bad_alloc
 * from the plan's buffers) become DK_ERR_ALLOC, so no exception leaves the
 * C ABI. */
int flush(dk_state *s)
{
	if (!s->pending)
		return DK_OK;
	try {
		return flush_queued(s);
	} catch (...) {
		return DK_ERR_ALLOC;
	}
}

static int flush_queued(dk_state *s)
{
	DK_TRACE();
	const unsigned n = s->n;
	const int prec = s->prec;
	const uint32_t cnt = s->pending->depth;
	std::vector<dk_flat_op> ops(cnt);
	{
		dk_op *o = s->pending;
		for (uint32_t i = 0; i < cnt; ++i, o = o->prev) {
			dk_flat_op &f = ops[cnt - 1 - i];
			f.gate = o->gate;
			f.k = o->k;
			memcpy(f.tg, o->tg, sizeof(f.tg));
			f.cm = o->cm;
			f.am = o->am;
		}
	}
	dk_plan_limits lim = {};
	lim.tile_bits = g.tile_bits;
	lim.fold = g.fold;
	/* one gate per sweep: nothing to fold into tensor-core products, and
	 * each sweep is a pure stream of the register, best on the scalar
	 * kernel with its 4 pinned low qubits (256-byte runs) */
	lim.tensor = g.fuse ? g.tensor : -1;
	dk_plan_default_limits(prec, n, &lim);
	lim.fuse = g.fuse;
	/* complex64 tensor sweeps of 12-bit tiles run on the tcgen05 kernel
	 * (whole columns per thread) unless DK_C64_TMEM=0 */
	lim.bank_mode = (prec == DK_C64 && dk::g_c64_tmem) ? 1 : 0;
	if (g.low_bits >= 0 && g.low_bits <= lim.tile_bits)
		lim.low_bits = g.low_bits;
	dk_plan plan;
	int rc = dk_plan_build(ops.data(), (int)cnt, n, prec, &lim, &plan);
	if (rc)
		return rc;

	/* device copy of the sweep programs and of generic-gate matrices */
	size_t gen_bytes = 0;
	for (int i = 0; i < plan.nsteps; ++i)
		if (plan.steps[i].kind == 2)
			gen_bytes += 16 * ops[plan.steps[i].op_index].gate->dim *
				     ops[plan.steps[i].op_index].gate->dim;
	const size_t blob_al = (plan.blob_bytes + 255) & ~(size_t)255;
	unsigned char *dblob = nullptr;
	rc = dev_alloc((void **)&dblob, blob_al + gen_bytes);
	if (rc) {
		dk_plan_free(&plan);
		return rc;
	}
	std::vector<size_t> gen_off(plan.nsteps, 0);
	{
		std::vector<unsigned char> host(blob_al + gen_bytes);
		if (plan.blob_bytes)
			memcpy(host.data(), plan.blob, plan.blob_bytes);
		size_t off = blob_al;
		for (int i = 0; i < plan.nsteps; ++i)
			if (plan.steps[i].kind == 2) {
				const dk_gate *gt = ops[plan.steps[i].op_index].gate;
				memcpy(host.data() + off, gt->m, 16 * gt->dim * gt->dim);
				gen_off[i] = off;
				off += 16 * gt->dim * gt->dim;
			}
		cudaError_t e = cudaMemcpyAsync(dblob, host.data(), host.size(),
						cudaMemcpyHostToDevice, CUR.st);
		if (e != cudaSuccess) {
			dev_free(dblob, blob_al + gen_bytes);
			dk_plan_free(&plan);
			return cuda_fail(e);
		}
		/* pageable source: the bytes are staged before the call returns, so
		 * `host` may be released without waiting for the stream */
		g.h2d += host.size();
	}

	dk_buf *src = s->buf;
	dk_buf *dst = src;
	if (src->refcount > 1) {
		rc = buf_new(n, prec, &dst);
		if (rc) {
			dev_free(dblob, blob_al + gen_bytes);
			dk_plan_free(&plan);
			return rc;
		}
	}
	const void *cur = src->d;
	const dk_scal *cur_sc = src->sc;
	for (int i = 0; i < plan.nsteps && rc == DK_OK; ++i) {
		const dk_step &stp = plan.steps[i];
		cudaError_t e;
		if (stp.kind == 1) {
			const dk_sweep_hdr *hp =
				(const dk_sweep_hdr *)(plan.blob + stp.prog_off);
			e = dk::launch_sweep(prec, cur, dst->d, dblob + stp.prog_off, hp,
					     cur_sc, dst->sc, CUR.scratch, g.num_sms, CUR.st);
			g.sweeps++;
			if (hp->mode == DK_SWEEP_TENSOR) {
				const dk_pass_desc *pd = (const dk_pass_desc *)(plan.blob +
										 stp.prog_off +
										 hp->pass_off);
				unsigned long long entries = 0;
				for (int p = 0; p < hp->npass; ++p)
					entries += (unsigned long long)(pd[p].g1 - pd[p].g0);
				g.mma_entry_amps += entries << n;
			}
			g.gates += (unsigned long long)stp.ngates;
		} else {
			const dk_flat_op &op = ops[stp.op_index];
			void *target = dst->d;
			void *tmp = nullptr;
			if (cur == dst->d) {
				rc = dev_alloc(&tmp, dst->bytes);
				if (rc)
					break;
				target = tmp;
			}
			e = dk::launch_generic_gate(prec, cur, target, n, op.k, op.tg,
						    op.cm, op.am,
						    (const double *)(dblob + gen_off[i]),
						    cur_sc, dst->sc, CUR.scratch, CUR.st);
			if (tmp) {
				dev_free(dst->d, dst->bytes);
				dst->d = tmp;
			}
			g.gates++;
		}
		if (e != cudaSuccess)
			rc = cuda_fail(e);
		cur = dst->d;
		cur_sc = dst->sc;
	}
	dev_free(dblob, blob_al + gen_bytes);
	dk_plan_free(&plan);
	if (rc) {
		if (dst != src)
			buf_release(dst);
		return rc;
	}
	if (dst != src) {
		buf_release(src);
		s->buf = dst;
	}
	op_release(s->pending);
	s->pending = nullptr;
	state_drop_caches(s);
	return DK_OK;
}

int read_scal(dk_state *s)
{
	if (s->have_norm)
		return DK_OK;
	dk_scal sc;
	CK(cudaMemcpyAsync(&sc, s->buf->sc, sizeof(sc), cudaMemcpyDeviceToHost, CUR.st));
	g.d2h += sizeof(sc);
	CK(cudaStreamSynchronize(CUR.st));
	/* a tcgen05 sweep whose bounded wait expired left the register's
	 * content undefined: report it instead of reading it */
	unsigned faults = 0;
	CK(dk::tm_fault_check(CUR.st, &faults));
	if (faults) {
		snprintf(g.err, sizeof(g.err), "tensor-memory sweep: %u bounded waits expired",
			 faults);
		return DK_ERR_TIMEOUT;
	}
	s->norm = sc.norm;
	s->csq = sc.csq;
	s->have_norm = 1;
	return DK_OK;
}

/* Ready a register for reading: live, non-empty, flushed, norm known. */
int prepare_read(dk_state *s)
{
	int rc = check_live(s);
	if (rc)
		return rc;
	if (s->n == 0 || !s->buf)
		return DK_ERR_EMPTY;
	rc = ensure_init();
	if (rc)
		return rc;
	rc = flush(s);
	if (rc)
		return rc;
	return read_scal(s);
}

int fill_hcache(dk_state *s)
{
	const uint64_t size = 1ull << s->n;
	double *h = (double *)malloc(16 * size);
	if (!h)
		return DK_ERR_ALLOC;
	double2 *tmp = nullptr;
	int rc = dev_alloc((void **)&tmp, 16 * size);
	if (rc) {
		free(h);
		return rc;
	}
	cudaError_t e = dk::launch_export(s->prec, s->buf->d, 0, size, tmp, CUR.st);
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(h, tmp, 16 * size, cudaMemcpyDeviceToHost, CUR.st);
	g.d2h += 16 * size;
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(CUR.st);
	dev_free(tmp, 16 * size);
	if (e != cudaSuccess) {
		free(h);
		return cuda_fail(e);
	}
	for (uint64_t i = 0; i < 2 * size; ++i)
		h[i] = h[i] / s->norm;
	s->hcache = h;
	return DK_OK;
}

int marginals_to_scratch(dk_state *s)
{
	if (s->have_marg) {
		CK(cudaMemcpyAsync(CUR.scratch.marg, s->marg, sizeof(double) * (s->n + 1),
				   cudaMemcpyHostToDevice, CUR.st));
		return DK_OK;
	}
	CK(dk::launch_marginals(s->prec, s->buf->d, s->n, CUR.scratch, CUR.st));
	return DK_OK;
}

} // namespace

/* ========================================================================== */

extern "C" {

const char *dk_strerror(int status)
{
	switch (status) {
	case DK_OK: return "ok";
	case DK_ERR_ALLOC: return "device memory allocation failed";
	case DK_ERR_QUBITS: return "Number of qubits exceeds maximum";
	case DK_ERR_ARG: return "invalid argument";
	case DK_ERR_CUDA: return "CUDA runtime error";
	case DK_ERR_BUDGET: return "device memory budget exceeded";
	case DK_ERR_TIMEOUT: return "device wait timed out";
	case DK_ERR_DEAD: return "registry was deleted";
	case DK_ERR_EMPTY: return "registry has no qubits";
	case DK_ERR_NORM0: return "New normalization constant is 0";
	case DK_ERR_NODEV: return "no CUDA device available";
	case DK_ERR_NOALLOC_LIMIT:
		return "register exceeds the allocation-free entry point's maximum of 40 qubits";
	default: return "unknown error";
	}
}

const char *dk_last_cuda_error(void) { return g.err; }

int dk_init(int device)
{
	DK_TRACE();
	std::lock_guard<std::mutex> lk(g.init_mu);
	if (g.inited.load())
		return DK_OK;
	int count = 0;
	if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
		cudaGetLastError();
		return DK_ERR_NODEV;
	}
	if (device < 0) {
		const char *env = getenv("DK_DEVICE");
		device = env ? atoi(env) : 0;
	}
	cudaError_t e = cudaSetDevice(device);
	if (e != cudaSuccess)
		return cuda_fail(e);
	g.device = device;
	e = cudaDeviceGetAttribute(&g.num_sms, cudaDevAttrMultiProcessorCount, device);
	if (e != cudaSuccess)
		return cuda_fail(e);
	cudaMemPool_t pool;
	if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
		uint64_t thr = UINT64_MAX;
		cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
	}
	int rc = create_slot(0);
	if (rc)
		return rc;
	g.nslots = 1;
	const char *b = getenv("DK_HBM_BUDGET_BYTES");
	g.budget = b ? (size_t)strtoull(b, nullptr, 10) : 0;
	const char *tb = getenv("DK_TILE_BITS");
	if (tb)
		g.tile_bits = atoi(tb);
	const char *f = getenv("DK_FUSE");
	if (f)
		g.fuse = atoi(f) ? 1 : 0;
	const char *fo = getenv("DK_FOLD");
	if (fo)
		g.fold = atoi(fo);
	const char *lb = getenv("DK_LOW_BITS");
	if (lb)
		g.low_bits = atoi(lb);
	const char *te = getenv("DK_TENSOR");
	if (te)
		g.tensor = atoi(te) ? 0 : -1;
	const char *tm = getenv("DK_C64_TMEM");
	if (tm)
		dk::g_c64_tmem = atoi(tm) ? 1 : 0;
	const char *tp = getenv("DK_C64_TMEM_PRESPLIT");
	if (tp)
		dk::g_tm_allow_presplit = atoi(tp) ? 1 : 0;
	g.inited = 1;
	return DK_OK;
}

int dk_slot_new(int *slot)
{
	if (!slot)
		return DK_ERR_ARG;
	int rc = ensure_init();
	if (rc)
		return rc;
	std::lock_guard<std::mutex> lk(g.slots_mu);
	const int id = g.nslots.load();
	if (id >= kMaxSlots)
		return DK_ERR_ARG;
	cudaSetDevice(g.device);
	rc = create_slot(id);
	if (rc)
		return rc;
	g.nslots = id + 1;
	*slot = id;
	return DK_OK;
}

int dk_slot_set(int slot)
{
	int rc = ensure_init();
	if (rc)
		return rc;
	if (slot < 0 || slot >= g.nslots.load())
		return DK_ERR_ARG;
	cudaSetDevice(g.device);
	t_slot = slot;
	return DK_OK;
}

int dk_slot_get(void) { return t_slot; }

int dk_gate_new(unsigned num_qubits, const double *matrix, dk_gate **out)
{
	if (!out || !matrix || num_qubits == 0 || num_qubits > DK_MAX_GATE_QUBITS)
		return DK_ERR_ARG;
	dk_gate *gt = (dk_gate *)calloc(1, sizeof(dk_gate));
	if (!gt)
		return DK_ERR_ALLOC;
	gt->refcount = 1;
	gt->k = num_qubits;
	gt->dim = 1ull << num_qubits;
	gt->m = (double *)malloc(16 * gt->dim * gt->dim);
	if (!gt->m) {
		free(gt);
		return DK_ERR_ALLOC;
	}
	memcpy(gt->m, matrix, 16 * gt->dim * gt->dim);
	*out = gt;
	return DK_OK;
}

int dk_gate_get(const dk_gate *gate, double *matrix)
{
	if (!gate || !matrix)
		return DK_ERR_ARG;
	memcpy(matrix, gate->m, 16 * gate->dim * gate->dim);
	return DK_OK;
}

unsigned dk_gate_num_qubits(const dk_gate *gate) { return gate ? gate->k : 0; }

void dk_gate_free(dk_gate *gate)
{
	if (!gate)
		return;
	if (__atomic_sub_fetch(&gate->refcount, 1, __ATOMIC_ACQ_REL) > 0)
		return;
	free(gate->m);
	free(gate);
}

int dk_state_new(unsigned num_qubits, int precision, dk_state **out)
{
	DK_TRACE();
	if (ensure_init() != DK_OK)
		return ensure_init();
	SlotLock lk(t_slot);
	if (!out || (precision != DK_C64 && precision != DK_C128))
		return DK_ERR_ARG;
	if (num_qubits == 0)
		return DK_ERR_ARG;
	if (num_qubits > DK_MAX_QUBITS)
		return DK_ERR_QUBITS;
	int rc = ensure_init();
	if (rc)
		return rc;
	dk_state *s = state_alloc(num_qubits, precision, t_slot);
	if (!s)
		return DK_ERR_ALLOC;
	rc = buf_new(num_qubits, precision, &s->buf);
	if (rc) {
		free(s);
		return rc;
	}
	cudaError_t e = dk::launch_init_zero(precision, s->buf->d, num_qubits,
					     s->buf->sc, CUR.st);
	if (e != cudaSuccess) {
		dk_state_free(s);
		return cuda_fail(e);
	}
	*out = s;
	return DK_OK;
}

int dk_state_from_host(unsigned num_qubits, int precision, const double *values,
		       dk_state **out)
{
	DK_TRACE();
	if (ensure_init() != DK_OK)
		return ensure_init();
	SlotLock lk(t_slot);
	if (!out || !values || (precision != DK_C64 && precision != DK_C128))
		return DK_ERR_ARG;
	if (num_qubits == 0)
		return DK_ERR_ARG;
	if (num_qubits > DK_MAX_QUBITS)
		return DK_ERR_QUBITS;
	int rc = ensure_init();
	if (rc)
		return rc;
	dk_state *s = state_alloc(num_qubits, precision, t_slot);
	if (!s)
		return DK_ERR_ALLOC;
	rc = buf_new(num_qubits, precision, &s->buf);
	if (rc) {
		free(s);
		return rc;
	}
	const size_t bytes = (size_t)16 << num_qubits;
	double *stage = (double *)s->buf->d;
	if (precision == DK_C64) {
		rc = dev_alloc((void **)&stage, bytes);
		if (rc) {
			dk_state_free(s);
			return rc;
		}
	}
	cudaError_t e = cudaMemcpyAsync(stage, values, bytes, cudaMemcpyHostToDevice, CUR.st);
	g.h2d += bytes;
	if (e == cudaSuccess)
		e = dk::launch_import(precision, stage, s->buf->d, num_qubits, s->buf->sc,
				      CUR.scratch, CUR.st);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(CUR.st);
	if (precision == DK_C64)
		dev_free(stage, bytes);
	if (e != cudaSuccess) {
		dk_state_free(s);
		return cuda_fail(e);
	}
	*out = s;
	return DK_OK;
}

int dk_state_clone(dk_state *src, dk_state **out)
{
	DK_TRACE();
	SlotLock lk(src ? src->slot : t_slot);
	int rc = check_live(src);
	if (rc)
		return rc;
	if (!out)
		return DK_ERR_ARG;
	dk_state *s = state_alloc(src->n, src->prec, src->slot);
	if (!s)
		return DK_ERR_ALLOC;
	s->buf = src->buf;
	if (s->buf)
		s->buf->refcount++;
	s->pending = src->pending;
	if (s->pending)
		s->pending->refcount++;
	*out = s;
	return DK_OK;
}

void dk_state_release(dk_state *s)
{
	if (!s)
		return;
	SlotLock lk(s->slot);
	buf_release(s->buf);
	s->buf = nullptr;
	op_release(s->pending);
	s->pending = nullptr;
	state_drop_caches(s);
	s->released = 1;
}

void dk_state_free(dk_state *s)
{
	if (!s)
		return;
	SlotLock lk(s->slot);
	buf_release(s->buf);
	op_release(s->pending);
	state_drop_caches(s);
	free(s);
}

size_t dk_state_mem_size(const dk_state *s)
{
	if (!s)
		return 0;
	size_t sz = sizeof(dk_state);
	if (s->buf)
		sz += s->buf->bytes + sizeof(dk_scal);
	return sz;
}

unsigned dk_state_num_qubits(const dk_state *s) { return s ? s->n : 0; }

int dk_state_precision(const dk_state *s) { return s ? s->prec : 0; }

int dk_apply_gate(dk_state *in, const dk_gate *gate, const unsigned *targets,
		  unsigned num_targets, const unsigned *controls,
		  unsigned num_controls, const unsigned *anticontrols,
		  unsigned num_anticontrols, dk_state **out)
{
	DK_TRACE();
	SlotLock lk(in ? in->slot : t_slot);
	int rc = check_live(in);
	if (rc)
		return rc;
	if (!gate || !out || (num_targets && !targets))
		return DK_ERR_ARG;
	if (in->n == 0 || !in->buf)
		return DK_ERR_EMPTY;
	if (num_targets != gate->k)
		return DK_ERR_ARG;
	uint64_t used = 0, cm = 0, am = 0;
	for (unsigned i = 0; i < num_targets; ++i) {
		if (targets[i] >= in->n || (used >> targets[i]) & 1u)
			return DK_ERR_ARG;
		used |= 1ull << targets[i];
	}
	for (unsigned i = 0; i < num_controls; ++i) {
		if (controls[i] >= in->n || (used >> controls[i]) & 1u)
			return DK_ERR_ARG;
		used |= 1ull << controls[i];
		cm |= 1ull << controls[i];
	}
	for (unsigned i = 0; i < num_anticontrols; ++i) {
		if (anticontrols[i] >= in->n || (used >> anticontrols[i]) & 1u)
			return DK_ERR_ARG;
		used |= 1ull << anticontrols[i];
		am |= 1ull << anticontrols[i];
	}
	dk_op *op = (dk_op *)calloc(1, sizeof(dk_op));
	if (!op)
		return DK_ERR_ALLOC;
	dk_state *s = state_alloc(in->n, in->prec, in->slot);
	if (!s) {
		free(op);
		return DK_ERR_ALLOC;
	}
	op->refcount = 1;
	op->gate = (dk_gate *)gate;
	gate_retain(op->gate);
	op->k = num_targets;
	for (unsigned i = 0; i < num_targets; ++i)
		op->tg[i] = targets[i];
	op->cm = cm;
	op->am = am;
	op->prev = in->pending;
	if (op->prev)
		op->prev->refcount++;
	op->depth = (op->prev ? op->prev->depth : 0) + 1;
	s->buf = in->buf;
	s->buf->refcount++;
	s->pending = op;
	*out = s;
	return DK_OK;
}

int dk_apply_gates(dk_state *in, unsigned count, const unsigned *op_k,
		   const unsigned *op_targets, const uint64_t *op_controls,
		   const uint64_t *op_anticontrols, const uint64_t *op_matrix,
		   const double *matrices, uint64_t num_matrix_entries, dk_state **out)
{
	DK_TRACE();
	if (!in || !out || (count && (!op_k || !op_targets || !op_controls || !op_anticontrols ||
				      !op_matrix || !matrices)))
		return DK_ERR_ARG;
	int rc = check_live(in);
	if (rc)
		return rc;
	if (in->n == 0 || !in->buf)
		return DK_ERR_EMPTY;
	const uint64_t full = (in->n >= 64) ? ~0ull : ((1ull << in->n) - 1ull);
	/* validate everything first: a failed call queues nothing */
	for (unsigned i = 0; i < count; ++i) {
		const unsigned k = op_k[i];
		if (k == 0 || k > 3)
			return DK_ERR_ARG;
		uint64_t used = 0;
		for (unsigned j = 0; j < k; ++j) {
			const unsigned t = op_targets[3 * i + j];
			if (t >= in->n || ((used >> t) & 1u))
				return DK_ERR_ARG;
			used |= 1ull << t;
		}
		const uint64_t cm = op_controls[i], am = op_anticontrols[i];
		if ((cm | am) & ~full || (cm & am) || ((cm | am) & used))
			return DK_ERR_ARG;
		if (op_matrix[i] > num_matrix_entries ||
		    (1ull << (2 * k)) > num_matrix_entries - op_matrix[i])
			return DK_ERR_ARG;
	}
	dk_state *cur = in;
	for (unsigned i = 0; i < count; ++i) {
		const unsigned k = op_k[i];
		dk_gate *g = nullptr;
		rc = dk_gate_new(k, matrices + 2 * op_matrix[i], &g);
		if (rc)
			break;
		unsigned ctl[64], act[64], nc = 0, na = 0;
		for (unsigned q = 0; q < in->n; ++q) {
			if ((op_controls[i] >> q) & 1u)
				ctl[nc++] = q;
			if ((op_anticontrols[i] >> q) & 1u)
				act[na++] = q;
		}
		dk_state *next = nullptr;
		rc = dk_apply_gate(cur, g, op_targets + 3 * i, k, ctl, nc, act, na, &next);
		dk_gate_free(g); /* the queued op keeps its own reference */
		if (rc)
			break;
		if (cur != in)
			dk_state_free(cur);
		cur = next;
	}
	if (rc) {
		if (cur != in)
			dk_state_free(cur);
		return rc;
	}
	if (cur == in)
		return dk_state_clone(in, out);
	*out = cur;
	return DK_OK;
}

int dk_state_norm(dk_state *s, double *norm, double *stored_norm)
{
	DK_TRACE();
	SlotLock lk(s ? s->slot : t_slot);
	int rc = prepare_read(s);
	if (rc)
		return rc;
	if (!norm || !stored_norm)
		return DK_ERR_ARG;
	*norm = s->norm;
	*stored_norm = sqrt(s->csq);
	return DK_OK;
}

int dk_state_read_half(dk_state *s, unsigned bit, int value, double scale, void *dst,
		       int on_device)
{
	DK_TRACE();
	SlotLock lk(s ? s->slot : t_slot);
	int rc = prepare_read(s);
	if (rc)
		return rc;
	if (!dst || bit >= s->n || (value != 0 && value != 1))
		return DK_ERR_ARG;
	const size_t bytes = amp_bytes(s->prec) << (s->n - 1);
	void *target = dst;
	if (!on_device) {
		rc = dev_alloc(&target, bytes);
		if (rc)
			return rc;
	}
	/* logical = stored / norm */
	cudaError_t e = dk::launch_read_half(s->prec, s->buf->d, s->n, bit, value,
					     scale / s->norm, target, CUR.st);
	if (!on_device) {
		if (e == cudaSuccess)
			e = cudaMemcpyAsync(dst, target, bytes, cudaMemcpyDeviceToHost, CUR.st);
		g.d2h += bytes;
		dev_free(target, bytes);
	}
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(CUR.st);
	return e == cudaSuccess ? DK_OK : cuda_fail(e);
}

int dk_state_replace_half(dk_state *in, unsigned bit, int value, double scale, const void *src,
			  int on_device, dk_state **out)
{
	DK_TRACE();
	SlotLock lk(in ? in->slot : t_slot);
	int rc = prepare_read(in);
	if (rc)
		return rc;
	if (!src || !out || bit >= in->n || (value != 0 && value != 1))
		return DK_ERR_ARG;
	const size_t bytes = amp_bytes(in->prec) << (in->n - 1);
	dk_state *s = state_alloc(in->n, in->prec, in->slot);
	if (!s)
		return DK_ERR_ALLOC;
	rc = buf_new(in->n, in->prec, &s->buf);
	if (rc) {
		free(s);
		return rc;
	}
	const void *from = src;
	void *stage = nullptr;
	cudaError_t e = cudaSuccess;
	if (!on_device) {
		rc = dev_alloc(&stage, bytes);
		if (rc) {
			dk_state_free(s);
			return rc;
		}
		e = cudaMemcpyAsync(stage, src, bytes, cudaMemcpyHostToDevice, CUR.st);
		g.h2d += bytes;
		from = stage;
	}
	if (e == cudaSuccess)
		e = dk::launch_replace_half(in->prec, in->buf->d, from, in->n, bit, value,
					    scale / in->norm, s->buf->d, s->buf->sc, CUR.scratch,
					    CUR.st);
	if (stage) {
		/* pageable source: the copy is staged before cudaMemcpyAsync
		 * returns; the kernel reads the device stage before the free */
		dev_free(stage, bytes);
	}
	if (e == cudaSuccess && !on_device)
		e = cudaStreamSynchronize(CUR.st);
	if (e != cudaSuccess) {
		dk_state_free(s);
		return cuda_fail(e);
	}
	*out = s;
	return DK_OK;
}

int dk_get_amplitude(dk_state *s, uint64_t id, double *re, double *im)
{
	DK_TRACE();
	SlotLock lk(s ? s->slot : t_slot);
	int rc = prepare_read(s);
	if (rc)
		return rc;
	if (!re || !im || id >= (1ull << s->n))
		return DK_ERR_ARG;
	if (!s->hcache && s->n <= 14) {
		rc = fill_hcache(s);
		if (rc)
			return rc;
	}
	if (s->hcache) {
		*re = s->hcache[2 * id];
		*im = s->hcache[2 * id + 1];
		return DK_OK;
	}
	double v[2];
	if (s->prec == DK_C128) {
		CK(cudaMemcpyAsync(v, (const double2 *)s->buf->d + id, 16,
				   cudaMemcpyDeviceToHost, CUR.st));
	} else {
		float f[2];
		CK(cudaMemcpyAsync(f, (const float2 *)s->buf->d + id, 8,
				   cudaMemcpyDeviceToHost, CUR.st));
		CK(cudaStreamSynchronize(CUR.st));
		v[0] = f[0];
		v[1] = f[1];
	}
	CK(cudaStreamSynchronize(CUR.st));
	*re = v[0] / s->norm;
	*im = v[1] / s->norm;
	return DK_OK;
}

int dk_get_amplitudes(dk_state *s, uint64_t first, uint64_t count, double *out)
{
	DK_TRACE();
	SlotLock lk(s ? s->slot : t_slot);
	int rc = prepare_read(s);
	if (rc)
		return rc;
	const uint64_t size = 1ull << s->n;
	if (!out || first > size || count > size - first)
		return DK_ERR_ARG;
	if (count == 0)
		return DK_OK;
	if (s->hcache) {
		memcpy(out, s->hcache + 2 * first, 16 * count);
		return DK_OK;
	}
	double2 *tmp = nullptr;
	rc = dev_alloc((void **)&tmp, 16 * count);
	if (rc)
		return rc;
	cudaError_t e = dk::launch_export(s->prec, s->buf->d, first, count, tmp, CUR.st);
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(out, tmp, 16 * count, cudaMemcpyDeviceToHost, CUR.st);
	g.d2h += 16 * count;
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(CUR.st);
	dev_free(tmp, 16 * count);
	if (e != cudaSuccess)
		return cuda_fail(e);
	for (uint64_t i = 0; i < 2 * count; ++i)
		out[i] = out[i] / s->norm;
	return DK_OK;
}

int dk_global_phase(dk_state *s, double *phase)
{
	DK_TRACE();
	SlotLock lk(s ? s->slot : t_slot);
	int rc = prepare_read(s);
	if (rc)
		return rc;
	if (!phase)
		return DK_ERR_ARG;
	if (s->have_phase) {
		*phase = s->phase;
		return DK_OK;
	}
	const uint64_t size = 1ull << s->n;
	uint64_t first = 0, chunk = 1ull << 16, found = UINT64_MAX;
	while (first < size) {
		const uint64_t cnt = chunk < size - first ? chunk : size - first;
		CK(dk::launch_first_nonzero(s->prec, s->buf->d, first, cnt, CUR.scratch,
					    CUR.st));
		unsigned long long hv = 0;
		CK(cudaMemcpyAsync(&hv, CUR.scratch.u64, 8, cudaMemcpyDeviceToHost, CUR.st));
		CK(cudaStreamSynchronize(CUR.st));
		if (hv != ~0ull) {
			found = hv;
			break;
		}
		first += cnt;
		chunk *= 4;
	}
	double ph = 0.0;
	if (found != UINT64_MAX) {
		double re, im;
		rc = dk_get_amplitude(s, found, &re, &im);
		if (rc)
			return rc;
		if (im != 0.0)
			ph = atan2(im, re);
	}
	s->phase = ph;
	s->have_phase = 1;
	*phase = ph;
	return DK_OK;
}

int dk_marginals(dk_state *s, double *p)
{
	DK_TRACE();
	SlotLock lk(s ? s->slot : t_slot);
	int rc = prepare_read(s);
	if (rc)
		return rc;
	if (!p)
		return DK_ERR_ARG;
	if (!s->have_marg) {
		double *m = (double *)malloc(sizeof(double) * (s->n + 1));
		if (!m)
			return DK_ERR_ALLOC;
		cudaError_t e = dk::launch_marginals(s->prec, s->buf->d, s->n, CUR.scratch, CUR.st);
		if (e == cudaSuccess)
			e = cudaMemcpyAsync(m, CUR.scratch.marg, sizeof(double) * (s->n + 1),
					    cudaMemcpyDeviceToHost, CUR.st);
		g.d2h += sizeof(double) * (s->n + 1);
		if (e == cudaSuccess)
			e = cudaStreamSynchronize(CUR.st);
		if (e != cudaSuccess) {
			free(m);
			return cuda_fail(e);
		}
		s->marg = m;
		s->have_marg = 1;
	}
	const double n2 = s->norm * s->norm;
	for (unsigned q = 0; q < s->n; ++q)
		p[q] = s->marg[q] / n2;
	return DK_OK;
}

int dk_probability(dk_state *s, unsigned target, double *p)
{
	DK_TRACE();
	SlotLock lk(s ? s->slot : t_slot);
	int rc = check_live(s);
	if (rc)
		return rc;
	if (!p || target >= s->n)
		return DK_ERR_ARG;
	double all[DK_MAX_QUBITS];
	rc = dk_marginals(s, all);
	if (rc)
		return rc;
	*p = all[target];
	return DK_OK;
}

int dk_measure_mask(dk_state *s, uint64_t mask, const double *rolls,
		    unsigned num_rolls, int8_t *results, dk_state **out)
{
	DK_TRACE();
	SlotLock lk(s ? s->slot : t_slot);
	int rc = prepare_read(s);
	if (rc)
		return rc;
	if (!results || !out)
		return DK_ERR_ARG;
	const unsigned n0 = s->n;
	const uint64_t full = (n0 >= 64) ? ~0ull : ((1ull << n0) - 1ull);
	unsigned need = (unsigned)__builtin_popcountll(mask & full);
	if (need > num_rolls || (need && !rolls))
		return DK_ERR_ARG;
	for (unsigned i = 0; i < need; ++i)
		if (!(rolls[i] >= 0.0 && rolls[i] < 1.0))
			return DK_ERR_ARG;
	for (unsigned i = 0; i < n0; ++i)
		results[i] = -1;
	if (need == 0)
		return dk_state_clone(s, out);

	if (need <= (unsigned)dk::kJointMaxQubits) {
		/* one pass: joint distribution of the measured qubits, outcomes
		 * decided on the device highest qubit first, one gather */
		double *rolls_dev = CUR.scratch.marg;
		int32_t *flags_dev = reinterpret_cast<int32_t *>(CUR.scratch.marg + 32);
		dk_buf *nb = nullptr;
		dk_scal *sel = nullptr;
		if (need < n0)
			rc = buf_new(n0 - need, s->prec, &nb);
		else
			rc = dev_alloc((void **)&sel, sizeof(dk_scal));
		if (rc)
			return rc;
		int32_t fl[64];
		cudaError_t e = cudaMemcpyAsync(rolls_dev, rolls, sizeof(double) * need,
						cudaMemcpyHostToDevice, CUR.st);
		g.h2d += sizeof(double) * need;
		if (e == cudaSuccess)
			e = dk::launch_measure_joint(s->prec, s->buf->d, nb ? nb->d : nullptr, n0,
						     mask & full, rolls_dev, flags_dev, s->buf->sc,
						     nb ? nb->sc : sel, CUR.scratch, CUR.st);
		if (e == cudaSuccess)
			e = cudaMemcpyAsync(fl, flags_dev, sizeof(int32_t) * need,
					    cudaMemcpyDeviceToHost, CUR.st);
		g.d2h += sizeof(int32_t) * need;
		dk_scal sc;
		memset(&sc, 0, sizeof(sc));
		if (e == cudaSuccess && nb)
			e = cudaMemcpyAsync(&sc, nb->sc, sizeof(sc), cudaMemcpyDeviceToHost, CUR.st);
		if (e == cudaSuccess)
			e = cudaStreamSynchronize(CUR.st);
		if (sel)
			dev_free(sel, sizeof(dk_scal));
		if (e != cudaSuccess) {
			if (nb)
				buf_release(nb);
			return cuda_fail(e);
		}
		if (nb && sc.zero_norm) {
			buf_release(nb);
			return DK_ERR_NORM0;
		}
		unsigned st = 0;
		for (unsigned i = 0; i < n0; ++i) {
			const unsigned q = n0 - i - 1;
			if ((mask >> q) & 1u)
				results[i] = (int8_t)fl[st++];
		}
		if (!nb) {
			*out = nullptr;
			return DK_OK;
		}
		dk_state *ns = state_alloc(n0 - need, s->prec, s->slot);
		if (!ns) {
			buf_release(nb);
			return DK_ERR_ALLOC;
		}
		ns->buf = nb;
		*out = ns;
		return DK_OK;
	}

	rc = marginals_to_scratch(s);
	if (rc)
		return rc;
	dk_buf *cur = s->buf;
	unsigned cur_n = n0;
	dk_buf *owned = nullptr; /* intermediate buffer we created */
	dk_scal *scratch_sc = nullptr;
	std::vector<int32_t> flags(n0, -1);
	unsigned rid = 0, left = need;
	for (unsigned i = 0; i < n0 && rc == DK_OK; ++i) {
		const unsigned q = n0 - i - 1;
		if (!((mask >> q) & 1u))
			continue;
		const double roll = rolls[rid++];
		left--;
		cudaError_t e;
		if (cur_n == 1) {
			if (!scratch_sc) {
				rc = dev_alloc((void **)&scratch_sc, sizeof(dk_scal));
				if (rc)
					break;
			}
			e = dk::launch_measure_collapse(cur->prec, cur->d, nullptr, 1, q, roll,
							-1, cur->sc, scratch_sc, CUR.scratch,
							CUR.st);
			if (e == cudaSuccess)
				e = cudaMemcpyAsync(&flags[i], &scratch_sc->flag, 4,
						    cudaMemcpyDeviceToHost, CUR.st);
			g.d2h += 4;
			if (e != cudaSuccess)
				rc = cuda_fail(e);
			if (owned)
				buf_release(owned);
			owned = nullptr;
			cur = nullptr;
			cur_n = 0;
			continue;
		}
		dk_buf *nb = nullptr;
		rc = buf_new(cur_n - 1, cur->prec, &nb);
		if (rc)
			break;
		e = dk::launch_measure_collapse(cur->prec, cur->d, nb->d, cur_n, q, roll,
						-1, cur->sc, nb->sc, CUR.scratch, CUR.st);
		if (e == cudaSuccess)
			e = cudaMemcpyAsync(&flags[i], &nb->sc->flag, 4,
					    cudaMemcpyDeviceToHost, CUR.st);
		g.d2h += 4;
		if (e == cudaSuccess && left > 0)
			e = dk::launch_marginals(nb->prec, nb->d, cur_n - 1, CUR.scratch, CUR.st);
		if (e != cudaSuccess) {
			rc = cuda_fail(e);
			buf_release(nb);
			break;
		}
		if (owned)
			buf_release(owned);
		owned = nb;
		cur = nb;
		cur_n--;
	}
	cudaError_t e = cudaStreamSynchronize(CUR.st);
	if (scratch_sc)
		dev_free(scratch_sc, sizeof(dk_scal));
	if (rc == DK_OK && e != cudaSuccess)
		rc = cuda_fail(e);
	int zero = 0;
	if (rc == DK_OK && owned) {
		dk_scal sc;
		e = cudaMemcpy(&sc, owned->sc, sizeof(sc), cudaMemcpyDeviceToHost);
		if (e != cudaSuccess)
			rc = cuda_fail(e);
		else
			zero = sc.zero_norm;
	}
	if (rc == DK_OK && zero)
		rc = DK_ERR_NORM0;
	if (rc) {
		if (owned)
			buf_release(owned);
		return rc;
	}
	for (unsigned i = 0; i < n0; ++i)
		results[i] = (int8_t)flags[i];
	if (cur_n == 0) {
		*out = nullptr;
		return DK_OK;
	}
	dk_state *ns = state_alloc(cur_n, s->prec, s->slot);
	if (!ns) {
		buf_release(owned);
		return DK_ERR_ALLOC;
	}
	ns->buf = owned;
	*out = ns;
	return DK_OK;
}

int dk_measure(dk_state *s, unsigned target, double roll, int *result,
	       dk_state **out)
{
	DK_TRACE();
	SlotLock lk(s ? s->slot : t_slot);
	int rc = check_live(s);
	if (rc)
		return rc;
	if (!result || !out || target >= s->n)
		return DK_ERR_ARG;
	std::vector<int8_t> res(s->n);
	rc = dk_measure_mask(s, 1ull << target, &roll, 1, res.data(), out);
	if (rc)
		return rc;
	*result = res[s->n - 1 - target];
	return DK_OK;
}

namespace {

/* The join itself, on most's slot (locked by the caller).  `ready`: an event
 * on least's stream that most's stream must wait for first (least was
 * flushed on its own slot), or NULL.  On success with a cross-slot join,
 * *done is an event recorded on most's stream after the join kernel. */
int join_on_most(dk_state *most, dk_state *least, cudaEvent_t ready, dk_state **out,
		 cudaEvent_t *done)
{
	int rc = prepare_read(most);
	if (rc == DK_OK && !ready)
		rc = prepare_read(least);
	if (ready && rc == DK_OK && cudaStreamWaitEvent(CUR.st, ready, 0) != cudaSuccess)
		rc = cuda_fail(cudaGetLastError());
	if (rc)
		return rc;
	if (!out || most->prec != least->prec)
		return DK_ERR_ARG;
	const unsigned n = most->n + least->n;
	if (n > DK_MAX_QUBITS)
		return DK_ERR_QUBITS;
	dk_state *s = state_alloc(n, most->prec, most->slot);
	if (!s)
		return DK_ERR_ALLOC;
	rc = buf_new(n, most->prec, &s->buf);
	if (rc) {
		free(s);
		return rc;
	}
	cudaError_t e = dk::launch_join(most->prec, most->buf->d, most->n, most->buf->sc,
					least->buf->d, least->n, least->buf->sc,
					s->buf->d, s->buf->sc, CUR.scratch, CUR.st);
	if (e == cudaSuccess && ready) {
		cudaEvent_t ev = nullptr;
		e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
		if (e == cudaSuccess) {
			e = cudaEventRecord(ev, CUR.st);
			if (e == cudaSuccess)
				*done = ev;
			else
				cudaEventDestroy(ev);
		}
		if (e != cudaSuccess) {
			/* no event to order least's stream by: the join kernel is
			 * queued, so wait for it here instead */
			cudaGetLastError();
			e = cudaStreamSynchronize(CUR.st);
		}
	}
	if (e != cudaSuccess) {
		dk_state_free(s);
		return cuda_fail(e);
	}
	*out = s;
	return DK_OK;
}

} // namespace

int dk_join(dk_state *most, dk_state *least, dk_state **out)
{
	DK_TRACE();
	if (!most || !least)
		return DK_ERR_ARG;
	int rc;
	cudaEvent_t ready = nullptr;
	if (least->slot != most->slot) {
		/* the least register is flushed on its own slot; most's slot waits */
		SlotLock lk2(least->slot);
		rc = prepare_read(least);
		if (rc)
			return rc;
		if (cudaEventCreateWithFlags(&ready, cudaEventDisableTiming) != cudaSuccess ||
		    cudaEventRecord(ready, CUR.st) != cudaSuccess) {
			if (ready)
				cudaEventDestroy(ready);
			return cuda_fail(cudaGetLastError());
		}
	}
	cudaEvent_t done = nullptr;
	{
		SlotLock lk(most->slot);
		rc = join_on_most(most, least, ready, out, &done);
	}
	if (ready)
		cudaEventDestroy(ready);
	if (done) {
		/* The join kernel reads least's buffer on most's stream.  Whatever
		 * least's slot queues next (freeing that buffer on its stream, or
		 * overwriting it in place when a register derived from least is
		 * flushed) waits for that read.  The two slot locks are taken one
		 * after the other, never nested, so joins in opposite directions
		 * cannot deadlock. */
		SlotLock lk2(least->slot);
		if (cudaStreamWaitEvent(CUR.st, done, 0) != cudaSuccess) {
			/* not ordered: wait for the join itself instead */
			cudaGetLastError();
			if (cudaEventSynchronize(done) != cudaSuccess && rc == DK_OK)
				rc = cuda_fail(cudaGetLastError());
		}
		cudaEventDestroy(done);
	}
	return rc;
}

int dk_reduced_density(dk_state *s, uint64_t keep_mask, double *out)
{
	DK_TRACE();
	SlotLock lk(s ? s->slot : t_slot);
	int rc = prepare_read(s);
	if (rc)
		return rc;
	const unsigned n = s->n;
	const uint64_t full = (n >= 64) ? ~0ull : ((1ull << n) - 1ull);
	if (!out || (keep_mask & ~full))
		return DK_ERR_ARG;
	const int k = __builtin_popcountll(keep_mask);
	if (k > 14)
		return DK_ERR_ARG;
	const uint64_t dim = 1ull << k;
	const uint64_t K = 1ull << (n - k);
	const bool direct = (s->prec == DK_C128) && (keep_mask == dim - 1);
	double2 *C = nullptr, *rho = nullptr, *M = nullptr;
	rc = dev_alloc((void **)&C, 16 * dim * dim);
	if (rc)
		return rc;
	rc = dev_alloc((void **)&rho, 16 * dim * dim);
	if (rc) {
		dev_free(C, 16 * dim * dim);
		return rc;
	}
	if (!direct) {
		rc = dev_alloc((void **)&M, 16ull << n);
		if (rc) {
			dev_free(C, 16 * dim * dim);
			dev_free(rho, 16 * dim * dim);
			return rc;
		}
	}
	cudaError_t e = cudaSuccess;
	const double2 *A = (const double2 *)s->buf->d;
	if (!direct) {
		e = dk::launch_gather_kept(s->prec, s->buf->d, n, keep_mask, M, CUR.st);
		A = M;
	}
	const double alpha = 1.0 / (s->norm * s->norm);
	/* tensor-core product X X^H, split over the traced index into partials
	 * that are added in a fixed order */
	const int ns = dk::rho_splits(dim, K, g.num_sms);
	double2 *part = nullptr;
	const size_t pbytes = (ns > 1 || dim < 64) ? 16 * dim * dim * (size_t)ns : 0;
	if (pbytes && dev_alloc((void **)&part, pbytes) != DK_OK) {
		dev_free(C, 16 * dim * dim);
		dev_free(rho, 16 * dim * dim);
		if (M)
			dev_free(M, 16ull << n);
		return DK_ERR_ALLOC;
	}
	if (e == cudaSuccess)
		e = dk::launch_rho(A, dim, K, alpha, ns, part, C, CUR.st);
	if (e == cudaSuccess)
		e = dk::launch_herm_fill(C, rho, dim, CUR.st);
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(out, rho, 16 * dim * dim, cudaMemcpyDeviceToHost, CUR.st);
	g.d2h += 16 * dim * dim;
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(CUR.st);
	dev_free(C, 16 * dim * dim);
	dev_free(rho, 16 * dim * dim);
	if (part)
		dev_free(part, pbytes);
	if (M)
		dev_free(M, 16ull << n);
	if (e != cudaSuccess)
		return cuda_fail(e);
	return DK_OK;
}

int dk_reduced_density_elem(dk_state *s, uint64_t keep_mask, uint64_t i,
			    uint64_t j, double *re, double *im)
{
	DK_TRACE();
	SlotLock lk(s ? s->slot : t_slot);
	int rc = prepare_read(s);
	if (rc)
		return rc;
	const unsigned n = s->n;
	const uint64_t full = (n >= 64) ? ~0ull : ((1ull << n) - 1ull);
	const int k = __builtin_popcountll(keep_mask);
	if (!re || !im || (keep_mask & ~full) || i >= (1ull << k) || j >= (1ull << k))
		return DK_ERR_ARG;
	double v[2];
	CK(dk::launch_rho_elem(s->prec, s->buf->d, n, keep_mask, i, j, s->buf->sc,
			       CUR.scratch, CUR.st));
	CK(cudaMemcpyAsync(v, CUR.scratch.marg, 16, cudaMemcpyDeviceToHost, CUR.st));
	CK(cudaStreamSynchronize(CUR.st));
	*re = v[0];
	*im = v[1];
	return DK_OK;
}

int dk_compare_states(dk_state *x, dk_state *y, double *fidelity, double *max_amp_err)
{
	DK_TRACE();
	if (!x || !y || x->n != y->n)
		return DK_ERR_ARG;
	if (x->slot != y->slot) {
		/* bring y up to date on its own slot first */
		SlotLock lk2(y->slot);
		int rc = prepare_read(y);
		if (rc)
			return rc;
		CK(cudaStreamSynchronize(CUR.st));
	}
	SlotLock lk(x->slot);
	int rc = prepare_read(x);
	if (rc == DK_OK)
		rc = prepare_read(y);
	if (rc)
		return rc;
	double v[3];
	CK(dk::launch_compare(x->prec, x->buf->d, 1.0 / x->norm, y->prec, y->buf->d, 1.0 / y->norm,
			      x->n, CUR.scratch, CUR.st));
	CK(cudaMemcpyAsync(v, CUR.scratch.marg, sizeof(v), cudaMemcpyDeviceToHost, CUR.st));
	CK(cudaStreamSynchronize(CUR.st));
	if (fidelity)
		*fidelity = v[0] * v[0] + v[1] * v[1];
	if (max_amp_err)
		*max_amp_err = v[2];
	return DK_OK;
}

int dk_set_fusion(int enable)
{
	
	g.fuse = enable ? 1 : 0;
	return DK_OK;
}

int dk_get_stats(uint64_t *kernel_launches, uint64_t *sweeps, uint64_t *gates_applied)
{
	
	if (kernel_launches)
		*kernel_launches = dk::g_launches;
	if (sweeps)
		*sweeps = g.sweeps;
	if (gates_applied)
		*gates_applied = g.gates;
	return DK_OK;
}

int dk_get_mma_stats(uint64_t *entry_amplitudes)
{
	if (entry_amplitudes)
		*entry_amplitudes = g.mma_entry_amps;
	return DK_OK;
}

int dk_get_tm_stats(uint64_t *presplit, uint64_t *per_entry)
{
	if (presplit)
		*presplit = dk::g_tm_presplit.load(std::memory_order_relaxed);
	if (per_entry)
		*per_entry = dk::g_tm_entry_b.load(std::memory_order_relaxed);
	return DK_OK;
}

int dk_get_io_stats(uint64_t *h2d_bytes, uint64_t *d2h_bytes)
{
	
	if (h2d_bytes)
		*h2d_bytes = g.h2d;
	if (d2h_bytes)
		*d2h_bytes = g.d2h;
	return DK_OK;
}

int dk_state_flush(dk_state *s)
{
	DK_TRACE();
	SlotLock lk(s ? s->slot : t_slot);
	int rc = check_live(s);
	if (rc)
		return rc;
	if (s->n == 0 || !s->buf)
		return DK_OK;
	rc = ensure_init();
	if (rc)
		return rc;
	return flush(s);
}

void *dk_stream(void)
{
	if (!g.inited.load())
		return nullptr;
	Slot *sl = g.slots[t_slot];
	return sl ? (void *)sl->st : nullptr;
}

int dk_sync(void)
{
	DK_TRACE();
	if (!g.inited.load())
		return DK_OK;
	const int ns = g.nslots.load();
	for (int i = 0; i < ns; ++i) {
		SlotLock lk(i);
		CK(cudaStreamSynchronize(CUR.st));
	}
	return DK_OK;
}

} // extern "C"
