/*
 * Batching form: thousands of independent registers (4-16 qubits), each with
 * its own gate sequence, executed by one persistent kernel per size class,
 * all captured in one CUDA graph.
 *
 * Every circuit is planned with the same planner as the plain path
 * (dk_plan.c): a register of n <= 12 qubits is one tile, so its whole program
 * runs on a shared-memory copy of the register (zero HBM traffic besides the
 * program and the results); a register of 13-16 qubits is owned by one thread
 * group that streams it through tiles of `tile_bits` qubits, sweep after sweep,
 * in a device buffer that stays L2-resident.  A thread group of 2^(m-3)
 * threads owns one register at a time (m = tile bits), several groups share a
 * 512-thread CTA and synchronise with their own barriers.  After the circuit
 * the group computes the register's reduced density matrix over its lower
 * `keep` qubits, renormalised by the trace as the reference's lazy norm does.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <memory>
#include <new>
#include <mutex>
#include <thread>
#include <vector>

#include "dk_device.cuh"
#include "dk_internal.h"
#include "dk_kernels.h"

/* Device descriptor of one register of a batch. */
typedef struct dk_breg {
	uint64_t prog; /* byte offset of its first sweep program in the blob */
	uint64_t state; /* amplitude offset of its buffer in the state array */
	uint64_t rho; /* complex offset of its reduced density matrix */
	uint32_t nsweep;
	uint32_t n;
	uint32_t keep;
	uint32_t pad;
} dk_breg;

namespace dk {
namespace {

constexpr int kBatchThreads = 512;

/* barrier over one register's thread group (G threads, group gid) */
__device__ __forceinline__ void group_sync(int G, int gid)
{
	if (G >= 64) {
		asm volatile("bar.sync %0, %1;\n" ::"r"(gid + 1), "r"(G) : "memory");
	} else if (G == 32) {
		__syncwarp();
	} else {
		const uint32_t lane = threadIdx.x & 31u;
		const uint32_t mask = ((1u << G) - 1u) << (lane & ~(uint32_t)(G - 1));
		__syncwarp(mask);
	}
}

/* Apply every pass of one sweep program to the group's shared tile. */
template <typename C2>
__device__ __forceinline__ void run_passes(C2 *tile, const unsigned char *prog,
					   const dk_sweep_hdr *h, uint32_t lt, uint64_t base,
					   int G, int gid)
{
	const dk_pass_desc *passes = reinterpret_cast<const dk_pass_desc *>(prog + h->pass_off);
	const uint4 *gates = reinterpret_cast<const uint4 *>(prog + h->gate_off);
	const dk_gate_cond *conds = reinterpret_cast<const dk_gate_cond *>(prog + h->cond_off);
	const C2 *mats = reinterpret_cast<const C2 *>(prog + h->mat_off);
	const int npass = h->npass;
	C2 a[NA];
	for (int p = 0; p < npass; ++p) {
		const dk_pass_desc *pd = passes + p;
		const uint32_t sgb = __ldg(&pd->slo[lt & 31]) ^ __ldg(&pd->shi[lt >> 5]);
		const uint32_t s0 = __ldg(&pd->sp[0]), s1 = __ldg(&pd->sp[1]), s2 = __ldg(&pd->sp[2]);
		uint32_t slot[NA];
#pragma unroll
		for (int r = 0; r < NA; ++r)
			slot[r] = sgb ^ ((r & 1) ? s0 : 0u) ^ ((r & 2) ? s1 : 0u) ^ ((r & 4) ? s2 : 0u);
#pragma unroll
		for (int r = 0; r < NA; ++r)
			a[r] = tile[slot[r]];
		PassCtx pc;
		if (__ldg(&pd->flags) & 1u) {
			pc.gb = __ldg(&pd->rlo[lt & 31]) | __ldg(&pd->rhi[lt >> 5]);
			pc.p0 = __ldg(&pd->pm[0]);
			pc.p1 = __ldg(&pd->pm[1]);
			pc.p2 = __ldg(&pd->pm[2]);
		} else {
			pc.gb = pc.p0 = pc.p1 = pc.p2 = 0;
		}
		const int g1 = __ldg(&pd->g1);
		for (int g = __ldg(&pd->g0); g < g1; ++g) {
			const uint4 d = __ldg(gates + g);
			const uint32_t gi = d.y & 0xffffu;
			if (gi != 0xffffu) {
				const uint64_t gc = __ldg(&conds[gi].gc), ga = __ldg(&conds[gi].ga);
				if (((base & gc) != gc) || (base & ga))
					continue;
			}
			apply_gate(a, pc, d.x & 0xffffu, d.y >> 16, d.z, d.w, mats + (d.x >> 16));
		}
#pragma unroll
		for (int r = 0; r < NA; ++r)
			tile[slot[r]] = a[r];
		group_sync(G, gid);
	}
}

template <typename R, int SW>
__global__ void __launch_bounds__(kBatchThreads, 1)
	k_batch(const unsigned char *__restrict__ blob, const dk_breg *__restrict__ regs,
		int nregs, int m, typename CT<R>::T *states, double2 *rho_out, int keep_states)
{
	typedef typename CT<R>::T C2;
	extern __shared__ __align__(16) unsigned char sm[];
	const int G = 1 << (m - PB);
	const int ngroups = blockDim.x / G;
	const int gid = threadIdx.x / G;
	const uint32_t lt = threadIdx.x % G;
	const uint32_t T = 1u << m;
	const int lanes = m - PB;
	C2 *tile = reinterpret_cast<C2 *>(sm) + (size_t)gid * T;
	double *red = reinterpret_cast<double *>(sm + (size_t)ngroups * T * sizeof(C2));

	for (int r = blockIdx.x * ngroups + gid; r < nregs; r += gridDim.x * ngroups) {
		const dk_breg reg = regs[r];
		const int n = (int)reg.n;
		const bool single = (n == m);
		C2 *gs = states + reg.state;
		const unsigned char *prog = blob + reg.prog;
		if (single) {
			/* |0..0>: the swizzle maps index 0 to slot 0 */
			for (uint32_t i = lt; i < T; i += G)
				tile[i] = mk((R)(i == 0 ? 1 : 0), (R)0);
			group_sync(G, gid);
		}
		for (uint32_t s = 0; s < reg.nsweep; ++s) {
			const dk_sweep_hdr *h = reinterpret_cast<const dk_sweep_hdr *>(prog);
			if (single) {
				run_passes(tile, prog, h, lt, 0, G, gid);
			} else {
				/* stream the register through tiles of this sweep's qubit set */
				uint64_t off_t = 0;
				for (int j = 0; j < lanes; ++j)
					if ((lt >> j) & 1u)
						off_t |= 1ull << h->qpos[j];
				uint64_t roff[NA];
#pragma unroll
				for (int rr = 0; rr < NA; ++rr) {
					uint64_t o = 0;
#pragma unroll
					for (int j = 0; j < PB; ++j)
						if ((rr >> j) & 1)
							o |= 1ull << h->qpos[lanes + j];
					roff[rr] = o;
				}
				const uint32_t stid = swz<SW>(lt);
				const uint64_t ntiles = h->ntiles;
				for (uint64_t t = 0; t < ntiles; ++t) {
					uint64_t base = t;
					for (int j = 0; j < m; ++j) {
						const int q = h->qpos[j];
						base = ((base >> q) << (q + 1)) | (base & ((1ull << q) - 1ull));
					}
					const uint64_t bo = base | off_t;
#pragma unroll
					for (int rr = 0; rr < NA; ++rr) {
						const uint64_t gi = bo | roff[rr];
						C2 v;
						if (s == 0)
							v = mk((R)(gi == 0 ? 1 : 0), (R)0);
						else
							v = gs[gi];
						tile[stid ^ swz<SW>((uint32_t)rr << lanes)] = v;
					}
					group_sync(G, gid);
					run_passes(tile, prog, h, lt, base, G, gid);
#pragma unroll
					for (int rr = 0; rr < NA; ++rr)
						gs[bo | roff[rr]] = tile[stid ^ swz<SW>((uint32_t)rr << lanes)];
					group_sync(G, gid);
				}
			}
			prog += h->bytes;
		}
		if (single && keep_states) {
			for (uint32_t i = lt; i < T; i += G)
				gs[i] = tile[swz<SW>(i)];
		}
		/* reduced density matrix of the lower `keep` qubits, divided by the
		 * trace (Sum |amp|^2), accumulated in FP64 */
		const uint32_t size = 1u << n;
		auto amp = [&](uint32_t i) -> double2 {
			return single ? to_c128(tile[swz<SW>(i)]) : to_c128(gs[i]);
		};
		double part = 0.0;
		for (uint32_t i = lt; i < size; i += G) {
			const double2 v = amp(i);
			part += v.x * v.x + v.y * v.y;
		}
		red[threadIdx.x] = part;
		group_sync(G, gid);
		if (lt == 0) {
			double t = 0.0;
			for (int i = 0; i < G; ++i)
				t += red[gid * G + i];
			red[gid * G] = t;
		}
		group_sync(G, gid);
		const double inv = 1.0 / red[gid * G];
		const int k = (int)reg.keep;
		const uint32_t dim = 1u << k, K = 1u << (n - k);
		double2 *ro = rho_out + reg.rho;
		for (uint32_t e = lt; e < dim * dim; e += G) {
			const uint32_t a0 = e >> k, a1 = e & (dim - 1u);
			double re = 0.0, im = 0.0;
			for (uint32_t b = 0; b < K; ++b) {
				const double2 x = amp((b << k) | a0), y = amp((b << k) | a1);
				re += x.x * y.x + x.y * y.y;
				im += x.y * y.x - x.x * y.y;
			}
			ro[e] = make_double2(re * inv, im * inv);
		}
		group_sync(G, gid);
	}
}

/* Per-register comparison of two batches of the same circuits (precision
 * form of the batch): fidelity |<x|y>|^2 / (<x|x> <y|y>) and the largest
 * |x_i / |x| - y_i / |y||, in FP64, one CTA per register (states in each
 * batch's own layout and precision; both offset tables are the same). */
template <typename CX, typename CY>
__global__ void __launch_bounds__(256)
	k_batch_compare(const CX *__restrict__ xs, const CY *__restrict__ ys,
			const uint64_t *__restrict__ offs, const uint32_t *__restrict__ ns,
			double *fid, double *err)
{
	const unsigned c = blockIdx.x;
	const uint64_t o = offs[c], cnt = 1ull << ns[c];
	double xr = 0.0, xi = 0.0, xx = 0.0, yy = 0.0;
	for (uint64_t i = threadIdx.x; i < cnt; i += blockDim.x) {
		const double2 x = to_c128(xs[o + i]), y = to_c128(ys[o + i]);
		xr += x.x * y.x + x.y * y.y; /* conj(x) y */
		xi += x.x * y.y - x.y * y.x;
		xx += sqabs(x);
		yy += sqabs(y);
	}
	__shared__ double red[4][256];
	red[0][threadIdx.x] = xr;
	red[1][threadIdx.x] = xi;
	red[2][threadIdx.x] = xx;
	red[3][threadIdx.x] = yy;
	__syncthreads();
	for (int st = blockDim.x >> 1; st > 0; st >>= 1) {
		if ((int)threadIdx.x < st)
			for (int k = 0; k < 4; ++k)
				red[k][threadIdx.x] += red[k][threadIdx.x + st];
		__syncthreads();
	}
	const double sx = 1.0 / sqrt(red[2][0]), sy = 1.0 / sqrt(red[3][0]);
	if (threadIdx.x == 0)
		fid[c] = (red[0][0] * red[0][0] + red[1][0] * red[1][0]) / (red[2][0] * red[3][0]);
	double m = 0.0;
	for (uint64_t i = threadIdx.x; i < cnt; i += blockDim.x) {
		const double2 x = to_c128(xs[o + i]), y = to_c128(ys[o + i]);
		const double dr = x.x * sx - y.x * sy, di = x.y * sx - y.y * sy;
		m = fmax(m, sqrt(dr * dr + di * di));
	}
	__syncthreads();
	red[0][threadIdx.x] = m;
	__syncthreads();
	for (int st = blockDim.x >> 1; st > 0; st >>= 1) {
		if ((int)threadIdx.x < st)
			red[0][threadIdx.x] = fmax(red[0][threadIdx.x], red[0][threadIdx.x + st]);
		__syncthreads();
	}
	if (threadIdx.x == 0) {
		err[c] = red[0][0];
	}
}

} // namespace
} // namespace dk

/* ========================================================================== */

namespace {

struct BatchClass {
	int m = 0;
	std::vector<dk_breg> regs;
	dk_breg *dregs = nullptr;
};

} // namespace

struct dk_batch {
	int prec = DK_C128;
	int tile_bits = 12;
	int ctas_per_sm = 1;
	int num_sms = 148;
	unsigned ncirc = 0;
	std::vector<uint64_t> rho_off, state_off;
	std::vector<unsigned> n, keep;
	std::vector<BatchClass> classes;
	unsigned char *dblob = nullptr;
	size_t blob_bytes = 0;
	void *dstates = nullptr;
	size_t state_amps = 0;
	double2 *drho = nullptr;
	size_t rho_elems = 0;
	cudaStream_t st = nullptr;
	std::vector<cudaStream_t> side;
	std::vector<cudaEvent_t> ev;
	cudaGraphExec_t graph = nullptr;
	int graph_keep_states = -1;
	/* host seconds of dk_batch_build: planning (all threads), assembling
	 * the program blob and register tables, device allocation and upload */
	double t_plan = 0.0, t_assemble = 0.0, t_upload = 0.0;
	char err[128] = { 0 };
};

/* fn(t, T) for t = 0 .. T-1, on T threads (the caller's included); shares
 * whose thread cannot be started run on the caller, so no exception leaves
 * this C-ABI library */
template <typename F> static void run_strided(unsigned T, F &fn)
{
	std::vector<std::thread> pool;
	std::vector<unsigned> inline_shares;
	for (unsigned t = 1; t < T; ++t) {
		try {
			pool.emplace_back(fn, t, T);
		} catch (...) {
			inline_shares.push_back(t);
		}
	}
	fn(0u, T);
	for (unsigned t : inline_shares)
		fn(t, T);
	for (auto &th : pool)
		th.join();
}

static int batch_cuda_fail(dk_batch *b, cudaError_t e)
{
	if (b)
		snprintf(b->err, sizeof(b->err), "%s", cudaGetErrorString(e));
	cudaGetLastError();
	return e == cudaErrorMemoryAllocation ? DK_ERR_ALLOC : DK_ERR_CUDA;
}

static void batch_release_device(dk_batch *b)
{
	if (b->graph)
		cudaGraphExecDestroy(b->graph);
	b->graph = nullptr;
	for (auto &c : b->classes)
		if (c.dregs)
			cudaFree(c.dregs);
	if (b->dblob)
		cudaFree(b->dblob);
	if (b->dstates)
		cudaFree(b->dstates);
	if (b->drho)
		cudaFree(b->drho);
	for (auto s : b->side)
		cudaStreamDestroy(s);
	for (auto e : b->ev)
		cudaEventDestroy(e);
	if (b->st)
		cudaStreamDestroy(b->st);
	b->side.clear();
	b->ev.clear();
	b->st = nullptr;
	b->dblob = nullptr;
	b->dstates = nullptr;
	b->drho = nullptr;
}

extern "C" {

static int batch_build(int precision, unsigned num_circuits, const unsigned *num_qubits,
		       const unsigned *keep_qubits, const uint64_t *op_start, const unsigned *op_k,
		       const unsigned *op_targets, const uint64_t *op_controls,
		       const uint64_t *op_anticontrols, const uint64_t *op_matrix,
		       const double *matrices, int tile_bits, int fold, dk_batch **out)
{
	if (!out || (precision != DK_C64 && precision != DK_C128) || !num_qubits ||
	    !keep_qubits || !op_start || (num_circuits == 0))
		return DK_ERR_ARG;
	if (tile_bits < 8 || tile_bits > 12)
		return DK_ERR_ARG;
	for (unsigned c = 0; c < num_circuits; ++c) {
		const unsigned n = num_qubits[c];
		if (n < 4 || n > 16 || keep_qubits[c] > n || keep_qubits[c] > 12 ||
		    op_start[c + 1] < op_start[c])
			return DK_ERR_ARG;
		for (uint64_t i = op_start[c]; i < op_start[c + 1]; ++i)
			if (op_k[i] == 0 || op_k[i] > 3)
				return DK_ERR_ARG;
	}
	int rc = dk_init(-1);
	if (rc)
		return rc;
	dk_batch *b = new dk_batch();
	b->prec = precision;
	b->tile_bits = tile_bits;
	b->ncirc = num_circuits;
	{
		int dev = 0;
		cudaGetDevice(&dev);
		cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, dev);
	}
	const size_t amp = precision == DK_C128 ? 16 : 8;
	std::unique_ptr<unsigned char[]> blob; /* programs, uninitialised between them */
	size_t blob_len = 0;
	std::vector<int> class_of_m(13, -1);
	b->rho_off.resize(num_circuits);
	b->state_off.resize(num_circuits);
	b->n.assign(num_qubits, num_qubits + num_circuits);
	b->keep.assign(keep_qubits, keep_qubits + num_circuits);

	/* Plan every circuit on its own (the planner is reentrant), on all host
	 * cores: circuit c goes to worker c mod T.  Each circuit's sweep
	 * programs are kept back to back in its own byte vector. */
	struct Planned {
		std::vector<unsigned char> prog;
		uint32_t nsweep = 0;
		int rc = 0;
	};
	std::vector<Planned> planned(num_circuits);
	auto plan_some = [&](unsigned first, unsigned stride) {
		std::vector<dk_gate> gates;
		std::vector<dk_flat_op> flat;
		for (unsigned c = first; c < num_circuits; c += stride) {
			Planned &pl = planned[c];
			const unsigned n = num_qubits[c];
			const uint64_t o0 = op_start[c], o1 = op_start[c + 1];
			try {
				gates.resize(o1 - o0);
				flat.resize(o1 - o0);
			} catch (...) {
				pl.rc = DK_ERR_ALLOC;
				continue;
			}
			for (uint64_t i = o0; i < o1; ++i) {
				dk_gate &gt = gates[i - o0];
				gt.refcount = 1;
				gt.k = op_k[i];
				gt.dim = 1ull << gt.k;
				gt.m = const_cast<double *>(matrices + 2 * op_matrix[i]);
				dk_flat_op &f = flat[i - o0];
				memset(&f, 0, sizeof(f));
				f.gate = &gt;
				f.k = gt.k;
				for (unsigned j = 0; j < gt.k && j < 3; ++j)
					f.tg[j] = op_targets[3 * i + j];
				f.cm = op_controls[i];
				f.am = op_anticontrols[i];
			}
			const int m = n <= 12 ? (int)n : tile_bits;
			dk_plan_limits lim = {};
			lim.tile_bits = m;
			lim.tensor = -1; /* the batch kernel runs scalar passes */
			lim.fold = fold;
			dk_plan_default_limits(precision, n, &lim);
			lim.tile_bits = m;
			if (lim.low_bits > m - 3)
				lim.low_bits = m - 3;
			dk_plan plan;
			pl.rc = dk_plan_build(flat.data(), (int)flat.size(), n, precision, &lim, &plan);
			if (pl.rc)
				continue;
			for (int st = 0; st < plan.nsteps && !pl.rc; ++st) {
				if (plan.steps[st].kind != 1) {
					pl.rc = DK_ERR_ARG; /* batches run sweepable gates only */
					break;
				}
				const dk_sweep_hdr *h =
					(const dk_sweep_hdr *)(plan.blob + plan.steps[st].prog_off);
				const size_t at = pl.prog.size();
				try {
					pl.prog.resize(at + h->bytes);
				} catch (...) {
					pl.rc = DK_ERR_ALLOC;
					break;
				}
				memcpy(pl.prog.data() + at, h, h->bytes);
				if (precision == DK_C64) {
					/* store the matrices in the amplitude precision, in place */
					dk_sweep_hdr *hh = (dk_sweep_hdr *)(pl.prog.data() + at);
					const double *src =
						(const double *)(pl.prog.data() + at + hh->mat_off);
					float *dst = (float *)(pl.prog.data() + at + hh->mat_off);
					const size_t nv = 2 * ((hh->bytes - hh->mat_off) / 16);
					for (size_t v = 0; v < nv; ++v)
						dst[v] = (float)src[v];
				}
			}
			pl.nsweep = (uint32_t)plan.nsteps;
			dk_plan_free(&plan);
		}
	};
	typedef std::chrono::steady_clock clk;
	const auto t0 = clk::now();
	unsigned T = std::thread::hardware_concurrency();
	if (T == 0)
		T = 1;
	if (T > 64)
		T = 64;
	if (T > num_circuits)
		T = num_circuits;
	{
		run_strided(T, plan_some);
	}
	const auto t1 = clk::now();
	for (unsigned c = 0; c < num_circuits; ++c)
		if (planned[c].rc) {
			rc = planned[c].rc;
			delete b;
			return rc;
		}
	/* each circuit's programs at a 16-byte aligned offset of one blob,
	 * copied in by all host threads */
	std::vector<size_t> at(num_circuits);
	for (unsigned c = 0; c < num_circuits; ++c) {
		const size_t pad = ((blob_len + 15) & ~(size_t)15) - blob_len;
		at[c] = blob_len + pad;
		blob_len = at[c] + planned[c].prog.size();
	}
	blob.reset(new (std::nothrow) unsigned char[blob_len ? blob_len : 16]);
	if (!blob) {
		delete b;
		return DK_ERR_ALLOC;
	}
	{
		auto copy_some = [&](unsigned first, unsigned stride) {
			for (unsigned c = first; c < num_circuits; c += stride) {
				if (!planned[c].prog.empty())
					memcpy(blob.get() + at[c], planned[c].prog.data(),
					       planned[c].prog.size());
				std::vector<unsigned char>().swap(planned[c].prog);
			}
		};
		run_strided(T, copy_some);
	}
	for (unsigned c = 0; c < num_circuits; ++c) {
		const unsigned n = num_qubits[c];
		const unsigned keep = keep_qubits[c];
		const int m = n <= 12 ? (int)n : tile_bits;
		dk_breg reg;
		memset(&reg, 0, sizeof(reg));
		reg.prog = at[c];
		reg.nsweep = planned[c].nsweep;
		reg.n = n;
		reg.keep = keep;
		reg.state = b->state_amps;
		reg.rho = b->rho_elems;
		b->state_off[c] = b->state_amps;
		b->rho_off[c] = b->rho_elems;
		b->state_amps += 1ull << n;
		b->rho_elems += 1ull << (2 * keep);
		if (class_of_m[m] < 0) {
			class_of_m[m] = (int)b->classes.size();
			b->classes.emplace_back();
			b->classes.back().m = m;
		}
		b->classes[class_of_m[m]].regs.push_back(reg);
	}
	/* larger registers first inside a class (better tail balance) */
	for (auto &cl : b->classes)
		std::stable_sort(cl.regs.begin(), cl.regs.end(),
				 [](const dk_breg &x, const dk_breg &y) { return x.n > y.n; });
	const auto t2 = clk::now();
	cudaError_t e = cudaMalloc(&b->dblob, blob_len ? blob_len : 16);
	if (e == cudaSuccess && blob_len)
		e = cudaMemcpy(b->dblob, blob.get(), blob_len, cudaMemcpyHostToDevice);
	b->blob_bytes = blob_len;
	if (e == cudaSuccess)
		e = cudaMalloc(&b->dstates, amp * b->state_amps);
	if (e == cudaSuccess)
		e = cudaMalloc(&b->drho, 16 * b->rho_elems);
	for (auto &cl : b->classes) {
		if (e != cudaSuccess)
			break;
		e = cudaMalloc(&cl.dregs, sizeof(dk_breg) * cl.regs.size());
		if (e == cudaSuccess)
			e = cudaMemcpy(cl.dregs, cl.regs.data(), sizeof(dk_breg) * cl.regs.size(),
				       cudaMemcpyHostToDevice);
	}
	if (e == cudaSuccess)
		e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking);
	for (size_t i = 0; e == cudaSuccess && i < b->classes.size(); ++i) {
		cudaStream_t s2;
		cudaEvent_t ev;
		e = cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking);
		if (e == cudaSuccess) {
			b->side.push_back(s2);
			e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
			if (e == cudaSuccess)
				b->ev.push_back(ev);
		}
	}
	if (e == cudaSuccess) {
		cudaEvent_t ev0;
		e = cudaEventCreateWithFlags(&ev0, cudaEventDisableTiming);
		if (e == cudaSuccess)
			b->ev.push_back(ev0);
	}
	if (e != cudaSuccess) {
		int r2 = batch_cuda_fail(b, e);
		batch_release_device(b);
		delete b;
		return r2;
	}
	const auto t3 = clk::now();
	b->t_plan = std::chrono::duration<double>(t1 - t0).count();
	b->t_assemble = std::chrono::duration<double>(t2 - t1).count();
	b->t_upload = std::chrono::duration<double>(t3 - t2).count();
	*out = b;
	return DK_OK;
}

int dk_batch_build(int precision, unsigned num_circuits, const unsigned *num_qubits,
		   const unsigned *keep_qubits, const uint64_t *op_start, const unsigned *op_k,
		   const unsigned *op_targets, const uint64_t *op_controls,
		   const uint64_t *op_anticontrols, const uint64_t *op_matrix,
		   const double *matrices, int tile_bits, int fold, dk_batch **out)
{
	DK_TRACE();
	/* host allocation failures (std::bad_alloc) become a status code */
	try {
		return batch_build(precision, num_circuits, num_qubits, keep_qubits, op_start, op_k,
				   op_targets, op_controls, op_anticontrols, op_matrix, matrices,
				   tile_bits, fold, out);
	} catch (...) {
		return DK_ERR_ALLOC;
	}
}

int dk_batch_set_ctas(dk_batch *b, int ctas_per_sm)
{
	if (!b || ctas_per_sm < 1 || ctas_per_sm > 4)
		return DK_ERR_ARG;
	b->ctas_per_sm = ctas_per_sm;
	if (b->graph) {
		cudaGraphExecDestroy(b->graph);
		b->graph = nullptr;
	}
	return DK_OK;
}

/* one tile per thread group: 512 threads x 8 amplitudes, plus the
 * per-thread reduction slots */
static size_t batch_smem(int prec, int m)
{
	const size_t amp = prec == DK_C128 ? 16 : 8;
	const int groups = dk::kBatchThreads >> (m - DK_PASS_BITS);
	return (size_t)groups * (amp << m) + sizeof(double) * dk::kBatchThreads;
}

static cudaError_t batch_enqueue(dk_batch *b, int keep_states)
{
	/* fork: every size class on its own stream, joined back on b->st */
	cudaEvent_t fork = b->ev.back();
	cudaError_t e = cudaEventRecord(fork, b->st);
	for (size_t i = 0; e == cudaSuccess && i < b->classes.size(); ++i) {
		const BatchClass &cl = b->classes[i];
		cudaStream_t s2 = b->side[i];
		e = cudaStreamWaitEvent(s2, fork, 0);
		if (e != cudaSuccess)
			break;
		const int G = 1 << (cl.m - DK_PASS_BITS);
		const int groups_per_cta = dk::kBatchThreads / G;
		const size_t smem = batch_smem(b->prec, cl.m);
		const int nregs = (int)cl.regs.size();
		int blocks = (nregs + groups_per_cta - 1) / groups_per_cta;
		const int cap = b->num_sms * b->ctas_per_sm;
		if (blocks > cap)
			blocks = cap;
		if (b->prec == DK_C128)
			dk::k_batch<double, 3><<<blocks, dk::kBatchThreads, smem, s2>>>(
				b->dblob, cl.dregs, nregs, cl.m, (double2 *)b->dstates, b->drho,
				keep_states);
		else
			dk::k_batch<float, 4><<<blocks, dk::kBatchThreads, smem, s2>>>(
				b->dblob, cl.dregs, nregs, cl.m, (float2 *)b->dstates, b->drho,
				keep_states);
		if (e == cudaSuccess)
			e = cudaGetLastError();
		if (e == cudaSuccess)
			e = cudaEventRecord(b->ev[i], s2);
		if (e == cudaSuccess)
			e = cudaStreamWaitEvent(b->st, b->ev[i], 0);
	}
	return e;
}

int dk_batch_run(dk_batch *b, int keep_states)
{
	DK_TRACE();
	if (!b)
		return DK_ERR_ARG;
	keep_states = keep_states ? 1 : 0;
	cudaError_t e = cudaSuccess;
	if (!b->graph || b->graph_keep_states != keep_states) {
		if (b->graph) {
			cudaGraphExecDestroy(b->graph);
			b->graph = nullptr;
		}
		const size_t smem = batch_smem(b->prec, 12);
		if (b->prec == DK_C128)
			e = cudaFuncSetAttribute(dk::k_batch<double, 3>,
						 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
		else
			e = cudaFuncSetAttribute(dk::k_batch<float, 4>,
						 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
		if (e != cudaSuccess)
			return batch_cuda_fail(b, e);
		cudaGraph_t g;
		e = cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal);
		if (e == cudaSuccess) {
			cudaError_t e2 = batch_enqueue(b, keep_states);
			e = cudaStreamEndCapture(b->st, &g);
			if (e2 != cudaSuccess)
				e = e2;
		}
		if (e == cudaSuccess) {
			e = cudaGraphInstantiate(&b->graph, g, 0);
			cudaGraphDestroy(g);
		}
		if (e != cudaSuccess)
			return batch_cuda_fail(b, e);
		b->graph_keep_states = keep_states;
	}
	e = cudaGraphLaunch(b->graph, b->st);
	if (e == cudaSuccess)
		dk::g_launches += b->classes.size();
	if (e != cudaSuccess)
		return batch_cuda_fail(b, e);
	return DK_OK;
}

int dk_batch_sync(dk_batch *b)
{
	DK_TRACE();
	if (!b)
		return DK_ERR_ARG;
	cudaError_t e = cudaStreamSynchronize(b->st);
	return e == cudaSuccess ? DK_OK : batch_cuda_fail(b, e);
}

void *dk_batch_stream(dk_batch *b) { return b ? (void *)b->st : nullptr; }

int dk_batch_rho(dk_batch *b, unsigned circuit, double *out)
{
	DK_TRACE();
	if (!b || !out || circuit >= b->ncirc)
		return DK_ERR_ARG;
	const size_t cnt = 1ull << (2 * b->keep[circuit]);
	cudaError_t e = cudaMemcpyAsync(out, b->drho + b->rho_off[circuit], 16 * cnt,
					cudaMemcpyDeviceToHost, b->st);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(b->st);
	return e == cudaSuccess ? DK_OK : batch_cuda_fail(b, e);
}

int dk_batch_rho_all(dk_batch *b, double *out, uint64_t *offsets)
{
	DK_TRACE();
	if (!b || !out)
		return DK_ERR_ARG;
	cudaError_t e = cudaMemcpyAsync(out, b->drho, 16 * b->rho_elems, cudaMemcpyDeviceToHost,
					b->st);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(b->st);
	if (offsets)
		for (unsigned c = 0; c < b->ncirc; ++c)
			offsets[c] = b->rho_off[c];
	return e == cudaSuccess ? DK_OK : batch_cuda_fail(b, e);
}

uint64_t dk_batch_rho_elems(const dk_batch *b) { return b ? b->rho_elems : 0; }

int dk_batch_state(dk_batch *b, unsigned circuit, double *out)
{
	DK_TRACE();
	if (!b || !out || circuit >= b->ncirc)
		return DK_ERR_ARG;
	const size_t cnt = 1ull << b->n[circuit];
	const size_t amp = b->prec == DK_C128 ? 16 : 8;
	std::vector<unsigned char> tmp(amp * cnt);
	cudaError_t e = cudaMemcpyAsync(tmp.data(), (unsigned char *)b->dstates + amp * b->state_off[circuit],
					amp * cnt, cudaMemcpyDeviceToHost, b->st);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(b->st);
	if (e != cudaSuccess)
		return batch_cuda_fail(b, e);
	if (b->prec == DK_C128) {
		memcpy(out, tmp.data(), 16 * cnt);
	} else {
		const float *f = (const float *)tmp.data();
		for (size_t i = 0; i < 2 * cnt; ++i)
			out[i] = f[i];
	}
	return DK_OK;
}

int dk_batch_compare(dk_batch *x, dk_batch *y, double *fidelity, double *max_amp_err)
{
	DK_TRACE();
	if (!x || !y || !fidelity || !max_amp_err || x->ncirc != y->ncirc || x->n != y->n ||
	    !x->dstates || !y->dstates)
		return DK_ERR_ARG;
	const unsigned nc = x->ncirc;
	/* both batches' work is done before the comparison reads them */
	cudaError_t e = cudaStreamSynchronize(y->st);
	uint64_t *doffs = nullptr;
	uint32_t *dns = nullptr;
	double *dout = nullptr;
	if (e == cudaSuccess)
		e = cudaMallocAsync(&doffs, sizeof(uint64_t) * nc, x->st);
	if (e == cudaSuccess)
		e = cudaMallocAsync(&dns, sizeof(uint32_t) * nc, x->st);
	if (e == cudaSuccess)
		e = cudaMallocAsync(&dout, 2 * sizeof(double) * nc, x->st);
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(doffs, x->state_off.data(), sizeof(uint64_t) * nc,
				    cudaMemcpyHostToDevice, x->st);
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(dns, x->n.data(), sizeof(uint32_t) * nc, cudaMemcpyHostToDevice,
				    x->st);
	if (e == cudaSuccess) {
		if (x->prec == DK_C64 && y->prec == DK_C128)
			dk::k_batch_compare<float2, double2><<<nc, 256, 0, x->st>>>(
				(const float2 *)x->dstates, (const double2 *)y->dstates, doffs, dns,
				dout, dout + nc);
		else if (x->prec == DK_C128 && y->prec == DK_C64)
			dk::k_batch_compare<double2, float2><<<nc, 256, 0, x->st>>>(
				(const double2 *)x->dstates, (const float2 *)y->dstates, doffs, dns,
				dout, dout + nc);
		else if (x->prec == DK_C64)
			dk::k_batch_compare<float2, float2><<<nc, 256, 0, x->st>>>(
				(const float2 *)x->dstates, (const float2 *)y->dstates, doffs, dns, dout,
				dout + nc);
		else
			dk::k_batch_compare<double2, double2><<<nc, 256, 0, x->st>>>(
				(const double2 *)x->dstates, (const double2 *)y->dstates, doffs, dns,
				dout, dout + nc);
		e = cudaGetLastError();
		dk::g_launches += 1;
	}
	std::vector<double> host(2 * (size_t)nc);
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(host.data(), dout, 2 * sizeof(double) * nc,
				    cudaMemcpyDeviceToHost, x->st);
	cudaFreeAsync(doffs, x->st);
	cudaFreeAsync(dns, x->st);
	cudaFreeAsync(dout, x->st);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(x->st);
	if (e != cudaSuccess)
		return batch_cuda_fail(x, e);
	memcpy(fidelity, host.data(), sizeof(double) * nc);
	memcpy(max_amp_err, host.data() + nc, sizeof(double) * nc);
	return DK_OK;
}

const char *dk_batch_error(const dk_batch *b) { return b ? b->err : ""; }

int dk_batch_build_times(const dk_batch *b, double *plan_s, double *assemble_s,
			 double *upload_s)
{
	if (!b)
		return DK_ERR_ARG;
	if (plan_s)
		*plan_s = b->t_plan;
	if (assemble_s)
		*assemble_s = b->t_assemble;
	if (upload_s)
		*upload_s = b->t_upload;
	return DK_OK;
}

void dk_batch_free(dk_batch *b)
{
	if (!b)
		return;
	if (b->st)
		cudaStreamSynchronize(b->st);
	batch_release_device(b);
	delete b;
}

} // extern "C"
