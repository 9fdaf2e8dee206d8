/*
 * Gate-fusion planner (host C).
 *
 * A queued run of gates (what the reference would apply one apply_gate call
 * at a time, qops.c:176-261) is cut into *sweeps*.  A sweep streams the whole
 * register through shared memory once, in tiles of 2^m amplitudes whose index
 * bits are a chosen qubit set Q (always containing the lowest `low_bits`
 * qubits so every tile is made of contiguous runs), and applies every gate
 * of the sweep to the tile.  A gate may join a sweep when its targets fit in
 * Q and it commutes with every earlier gate left for a later sweep (disjoint
 * supports).  Controls need not be in Q: those outside Q are constant over a
 * tile and become a per-tile predicate.
 *
 * Inside a sweep the gates are grouped into *passes*: each pass gathers, per
 * thread, the 8 amplitudes that differ in 3 chosen tile bits into registers
 * and applies every gate of the pass whose targets lie in those bits.
 *
 * Gates on more than 3 qubits, and dense (non-diagonal) 3-qubit gates, become
 * generic single-gate steps.
 */
#include <stdlib.h>
#include <string.h>

#include "dk_internal.h"

static int popc(uint64_t x) { return __builtin_popcountll(x); }

/* gates examined per pass when grouping a sweep's gates into passes */
#define DK_PASS_WINDOW 64

void dk_plan_default_limits(int prec, unsigned n, dk_plan_limits *lim)
{
	int m = (prec == DK_C64) ? DK_TILE_BITS_C64 : DK_TILE_BITS_C128;
	if (lim->tile_bits >= DK_PASS_BITS && lim->tile_bits <= 12)
		m = lim->tile_bits; /* caller's choice */
	if ((int)n < m)
		m = (int)n;
	lim->tile_bits = m;
	lim->low_bits = m < 4 ? m : 4;
	lim->max_gates = 512;
	lim->max_passes = 512;
	lim->max_mat = 4096; /* complex entries: <= 64 KiB of a sweep's shared memory */
	lim->fuse = 1;
}

/* Kind of a gate as executed by the sweep kernel. */
int dk_gate_classify(const struct dk_gate *g)
{
	const uint64_t d = g->dim;
	int offzero = 1, diagzero = 1;
	for (uint64_t r = 0; r < d; r++)
		for (uint64_t c = 0; c < d; c++) {
			const double *e = g->m + 2 * (r * d + c);
			int z = (e[0] == 0.0 && e[1] == 0.0);
			if (r == c)
				diagzero &= z;
			else
				offzero &= z;
		}
	if (g->k == 1) {
		const double *m = g->m;
		if (offzero) {
			if (m[0] == 1.0 && m[1] == 0.0 && m[6] == -1.0 && m[7] == 0.0)
				return DK_GK_NEG1;
			if (m[0] == 1.0 && m[1] == 0.0)
				return DK_GK_PHASE1;
			return DK_GK_DIAG1;
		}
		if (diagzero) {
			if (m[2] == 1.0 && m[3] == 0.0 && m[4] == 1.0 && m[5] == 0.0)
				return DK_GK_SWAP1;
			return DK_GK_ANTI1;
		}
		return DK_GK_DENSE1;
	}
	if (offzero)
		return DK_GK_DIAGK;
	return g->k == 2 ? DK_GK_DENSE2 : DK_GK_DENSE3;
}

static uint64_t support(const dk_flat_op *op)
{
	uint64_t s = op->cm | op->am;
	for (unsigned i = 0; i < op->k; i++)
		s |= UINT64_C(1) << op->tg[i];
	return s;
}

static uint64_t target_mask(const dk_flat_op *op)
{
	uint64_t s = 0;
	for (unsigned i = 0; i < op->k; i++)
		s |= UINT64_C(1) << op->tg[i];
	return s;
}

static int mat_entries(int kind, unsigned k)
{
	switch (kind) {
	case DK_GK_SWAP1:
	case DK_GK_NEG1:
		return 0;
	case DK_GK_PHASE1:
		return 1;
	case DK_GK_DIAG1:
	case DK_GK_ANTI1:
		return 2;
	case DK_GK_DIAGK:
		return 1 << k;
	default:
		return 1 << (2 * k);
	}
}

typedef struct blob_t {
	unsigned char *p;
	size_t len, cap;
} blob_t;

static int blob_reserve(blob_t *b, size_t extra)
{
	if (b->len + extra <= b->cap)
		return 0;
	size_t nc = b->cap ? b->cap : 4096;
	while (nc < b->len + extra)
		nc *= 2;
	unsigned char *np = (unsigned char *)realloc(b->p, nc);
	if (!np)
		return -1;
	b->p = np;
	b->cap = nc;
	return 0;
}

static size_t align_up(size_t x, size_t a) { return (x + a - 1) & ~(a - 1); }

/* Lane mapping: thread-index bits -> the non-pass tile bits, ordered so the
 * lowest `res` thread bits land on tile bits with pairwise distinct residues
 * mod `res` (then the XOR swizzle of the shared tile makes each quarter-warp
 * (complex128) / half-warp (complex64) access bank-conflict free). */
static int lane_map(int m, const uint8_t *pb, int res, uint8_t *lane)
{
	int used[64] = { 0 };
	int free_bits[64], nf = 0, nl = 0;
	for (int j = 0; j < DK_PASS_BITS; j++)
		used[pb[j]] = 1;
	for (int b = 0; b < m; b++)
		if (!used[b])
			free_bits[nf++] = b;
	int taken[64] = { 0 };
	for (int r = 0; r < res && nl < nf; r++) {
		for (int i = 0; i < nf; i++) {
			if (!taken[i] && free_bits[i] % res == r) {
				lane[nl++] = (uint8_t)free_bits[i];
				taken[i] = 1;
				break;
			}
		}
	}
	for (int i = 0; i < nf; i++)
		if (!taken[i])
			lane[nl++] = (uint8_t)free_bits[i];
	return nl;
}

/* The tile swizzle (must equal the kernel's swz<SW>): the low SW bits of the
 * slot are XORed with every higher SW-bit group. */
static uint32_t swizzle(uint32_t i, int sw)
{
	uint32_t f = 0;
	for (int s = sw; s < 20; s += sw)
		f ^= i >> s;
	return i ^ (f & ((1u << sw) - 1u));
}

static void pass_tables(dk_pass_desc *pd, const uint8_t *pb, int m, int sw)
{
	uint8_t lane[32];
	const int nl = lane_map(m, pb, sw, lane);
	for (int j = 0; j < DK_PASS_BITS; j++) {
		pd->pm[j] = 1u << pb[j];
		pd->sp[j] = swizzle(pd->pm[j], sw);
	}
	for (uint32_t x = 0; x < 32; x++) {
		uint32_t raw = 0;
		for (int j = 0; j < 5 && j < nl; j++)
			if ((x >> j) & 1u)
				raw |= 1u << lane[j];
		pd->rlo[x] = raw;
		pd->slo[x] = swizzle(raw, sw);
	}
	for (uint32_t y = 0; y < 16; y++) {
		uint32_t raw = 0;
		for (int j = 0; j < 4 && 5 + j < nl; j++)
			if ((y >> j) & 1u)
				raw |= 1u << lane[5 + j];
		pd->rhi[y] = raw;
		pd->shi[y] = swizzle(raw, sw);
	}
}

/* Emit one sweep program for ops[idx[0..cnt)] over tile set Q. */
static int emit_sweep(blob_t *b, const dk_flat_op *ops, const int *idx,
		      int cnt, uint64_t Q, unsigned n, int prec, int m,
		      const int *kinds, dk_step *step)
{
	uint8_t qpos[64];
	int8_t loc_of[64];
	int nq = 0;
	memset(loc_of, -1, sizeof(loc_of));
	for (unsigned q = 0; q < n; q++)
		if (Q & (UINT64_C(1) << q)) {
			loc_of[q] = (int8_t)nq;
			qpos[nq++] = (uint8_t)q;
		}
	if (nq != m)
		return -1;

	/* group the sweep's gates into passes (commutation-aware greedy) */
	int *rem = (int *)malloc(sizeof(int) * (cnt ? cnt : 1));
	int *defer = (int *)malloc(sizeof(int) * (cnt ? cnt : 1));
	int *order = (int *)malloc(sizeof(int) * (cnt ? cnt : 1));
	dk_pass_desc *passes =
		(dk_pass_desc *)calloc((size_t)(cnt ? cnt : 1), sizeof(dk_pass_desc));
	uint8_t(*pbits)[DK_PASS_BITS] =
		(uint8_t(*)[DK_PASS_BITS])calloc((size_t)(cnt ? cnt : 1), DK_PASS_BITS);
	if (!rem || !defer || !order || !passes || !pbits) {
		free(rem);
		free(defer);
		free(order);
		free(passes);
		free(pbits);
		return -1;
	}
	int nrem = cnt, npass = 0, nord = 0;
	for (int i = 0; i < cnt; i++)
		rem[i] = idx[i];
	const int res = (prec == DK_C64) ? 4 : 3;
	while (nrem > 0) {
		uint32_t P = 0;
		uint64_t blocked = 0;
		int nd = 0;
		dk_pass_desc *pd = &passes[npass];
		pd->g0 = (uint16_t)nord;
		for (int i = 0; i < nrem; i++) {
			const dk_flat_op *op = &ops[rem[i]];
			uint64_t sup = support(op);
			/* bounded lookahead keeps grouping linear in the gate count */
			if (i >= DK_PASS_WINDOW || (sup & blocked)) {
				defer[nd++] = rem[i];
				blocked |= sup;
				continue;
			}
			uint32_t tl = 0;
			for (unsigned t = 0; t < op->k; t++)
				tl |= 1u << loc_of[op->tg[t]];
			if (popc(P | tl) <= DK_PASS_BITS) {
				P |= tl;
				order[nord++] = rem[i];
			} else {
				defer[nd++] = rem[i];
				blocked |= sup;
			}
		}
		pd->g1 = (uint16_t)nord;
		/* fill the pass up to DK_PASS_BITS bits with the highest free tile bits */
		for (int bit = m - 1; popc(P) < DK_PASS_BITS && bit >= 0; bit--)
			P |= 1u << bit;
		int j = 0;
		for (int bit = 0; bit < m; bit++)
			if (P & (1u << bit))
				pbits[npass][j++] = (uint8_t)bit;
		pass_tables(pd, pbits[npass], m, res);
		for (int g = pd->g0; g < pd->g1; g++) {
			const dk_flat_op *op = &ops[order[g]];
			if ((op->cm | op->am) & Q)
				pd->flags |= 1u;
		}
		npass++;
		memcpy(rem, defer, sizeof(int) * (size_t)nd);
		nrem = nd;
	}

	/* size the program */
	int nmat = 0;
	for (int i = 0; i < nord; i++)
		nmat += mat_entries(kinds[order[i]], ops[order[i]].k);
	int ncond = 0;
	for (int i = 0; i < nord; i++) {
		const dk_flat_op *op = &ops[order[i]];
		if ((op->cm | op->am) & ~Q)
			ncond++;
	}
	size_t pass_off = align_up(sizeof(dk_sweep_hdr), 16);
	size_t gate_off = align_up(pass_off + sizeof(dk_pass_desc) * (size_t)npass, 16);
	size_t cond_off = align_up(gate_off + sizeof(dk_gate_desc) * (size_t)nord, 16);
	size_t mat_off = align_up(cond_off + sizeof(dk_gate_cond) * (size_t)ncond, 16);
	size_t bytes = align_up(mat_off + 16 * (size_t)nmat, 16);

	size_t start = align_up(b->len, 16);
	if (blob_reserve(b, (start - b->len) + bytes)) {
		free(rem);
		free(defer);
		free(order);
		free(passes);
		free(pbits);
		return -1;
	}
	memset(b->p + b->len, 0, (start - b->len) + bytes);
	b->len = start;
	unsigned char *base = b->p + start;
	dk_sweep_hdr *h = (dk_sweep_hdr *)base;
	h->m = m;
	h->n = (int32_t)n;
	h->npass = npass;
	h->ngate = nord;
	h->ntiles = UINT64_C(1) << (n - (unsigned)m);
	memcpy(h->qpos, qpos, (size_t)m);
	h->pass_off = (uint32_t)pass_off;
	h->gate_off = (uint32_t)gate_off;
	h->mat_off = (uint32_t)mat_off;
	h->bytes = (uint32_t)bytes;
	h->cond_off = (uint32_t)cond_off;
	h->ncond = (uint32_t)ncond;
	memcpy(base + pass_off, passes, sizeof(dk_pass_desc) * (size_t)npass);

	dk_gate_desc *gd = (dk_gate_desc *)(base + gate_off);
	dk_gate_cond *conds = (dk_gate_cond *)(base + cond_off);
	double *mats = (double *)(base + mat_off);
	int moff = 0, all_touched = 0, ci = 0;
	int pi = 0;
	for (int i = 0; i < nord; i++) {
		while (pi < npass && i >= passes[pi].g1)
			pi++;
		const dk_flat_op *op = &ops[order[i]];
		const int kind = kinds[order[i]];
		dk_gate_desc *g = &gd[i];
		uint8_t treg[3] = { 0, 0, 0 };
		for (unsigned t = 0; t < op->k; t++) {
			int lb = loc_of[op->tg[t]];
			for (int r = 0; r < DK_PASS_BITS; r++)
				if (pbits[pi][r] == lb)
					treg[t] = (uint8_t)r;
		}
		uint64_t gc = 0, ga = 0;
		for (unsigned q = 0; q < n; q++) {
			uint64_t bit = UINT64_C(1) << q;
			if (op->cm & bit) {
				if (loc_of[q] >= 0)
					g->lc |= 1u << loc_of[q];
				else
					gc |= bit;
			}
			if (op->am & bit) {
				if (loc_of[q] >= 0)
					g->la |= 1u << loc_of[q];
				else
					ga |= bit;
			}
		}
		if (gc == 0 && ga == 0) {
			all_touched = 1;
			g->gcond = 0xffff;
		} else {
			conds[ci].gc = gc;
			conds[ci].ga = ga;
			g->gcond = (uint16_t)ci++;
		}
		const int ctl = (g->lc | g->la) != 0;
		switch (kind) {
		case DK_GK_DENSE1: g->code = (uint16_t)(DK_GC_DENSE1 + treg[0] + 3 * ctl); break;
		case DK_GK_SWAP1: g->code = (uint16_t)(DK_GC_SWAP1 + treg[0] + 3 * ctl); break;
		case DK_GK_PHASE1: g->code = (uint16_t)(DK_GC_PHASE1 + treg[0] + 3 * ctl); break;
		case DK_GK_DIAG1: g->code = (uint16_t)(DK_GC_DIAG1 + treg[0] + 3 * ctl); break;
		case DK_GK_ANTI1: g->code = (uint16_t)(DK_GC_ANTI1 + treg[0] + 3 * ctl); break;
		case DK_GK_NEG1: g->code = (uint16_t)(DK_GC_NEG1 + treg[0] + 3 * ctl); break;
		case DK_GK_DENSE2: {
			static const int pair_index[3][3] = { { -1, 0, 1 }, { 2, -1, 3 }, { 4, 5, -1 } };
			g->code = (uint16_t)(DK_GC_DENSE2 + pair_index[treg[0]][treg[1]]);
			break;
		}
		default: g->code = DK_GC_DIAGK; break;
		}
		g->info = (uint16_t)(treg[0] | (treg[1] << 2) | (treg[2] << 4) |
				     ((op->k & 3u) << 6) | ((unsigned)kind << 8));
		g->mat = (uint16_t)moff;
		const double *src = op->gate->m;
		const uint64_t d = op->gate->dim;
		double *dst = mats + 2 * moff;
		switch (kind) {
		case DK_GK_SWAP1:
		case DK_GK_NEG1:
			break;
		case DK_GK_PHASE1:
			memcpy(dst, src + 2 * 3, 16);
			break;
		case DK_GK_DIAG1:
			memcpy(dst, src, 16);
			memcpy(dst + 2, src + 2 * 3, 16);
			break;
		case DK_GK_ANTI1:
			memcpy(dst, src + 2 * 1, 16);
			memcpy(dst + 2, src + 2 * 2, 16);
			break;
		case DK_GK_DIAGK:
			for (uint64_t r = 0; r < d; r++)
				memcpy(dst + 2 * r, src + 2 * (r * d + r), 16);
			break;
		default:
			memcpy(dst, src, 16 * d * d);
		}
		moff += mat_entries(kind, op->k);
	}
	h->all_touched = all_touched;
	b->len = start + bytes;
	step->kind = 1;
	step->prog_off = start;
	step->op_index = -1;
	step->ngates = nord;
	free(rem);
	free(defer);
	free(order);
	free(passes);
	free(pbits);
	return 0;
}

int dk_plan_build(const dk_flat_op *ops, int nops, unsigned n, int prec,
		  const dk_plan_limits *lim, dk_plan *plan)
{
	memset(plan, 0, sizeof(*plan));
	if (nops <= 0)
		return 0;
	blob_t b = { 0, 0, 0 };
	int *rem = (int *)malloc(sizeof(int) * (size_t)nops);
	int *defer = (int *)malloc(sizeof(int) * (size_t)nops);
	int *take = (int *)malloc(sizeof(int) * (size_t)nops);
	int *kinds = (int *)malloc(sizeof(int) * (size_t)nops);
	dk_step *steps = (dk_step *)calloc((size_t)nops, sizeof(dk_step));
	if (!rem || !defer || !take || !kinds || !steps)
		goto fail;
	const int m = lim->tile_bits;
	const int sweepable = (m >= DK_PASS_BITS);
	for (int i = 0; i < nops; i++) {
		rem[i] = i;
		kinds[i] = (ops[i].k <= DK_SWEEP_MAX_K && sweepable)
				   ? dk_gate_classify(ops[i].gate)
				   : 0;
		/* dense 3-qubit gates run as generic steps (kept out of the
		 * register budget of the sweep) */
		if (kinds[i] == DK_GK_DENSE3)
			kinds[i] = 0;
	}
	int nrem = nops, nsteps = 0;
	while (nrem > 0) {
		/* a leading gate the sweep cannot run becomes a generic step */
		if (kinds[rem[0]] == 0) {
			steps[nsteps].kind = 2;
			steps[nsteps].op_index = rem[0];
			steps[nsteps].ngates = 1;
			nsteps++;
			memmove(rem, rem + 1, sizeof(int) * (size_t)(nrem - 1));
			nrem--;
			continue;
		}
		/* pinned low qubits leave room for any gate the sweep can run */
		int low = lim->low_bits;
		if (low > m - DK_SWEEP_MAX_K)
			low = m - DK_SWEEP_MAX_K;
		uint64_t Q = 0;
		for (int q = 0; q < low; q++)
			Q |= UINT64_C(1) << q;
		uint64_t blocked = 0;
		int nd = 0, nt = 0, nmat = 0;
		for (int i = 0; i < nrem; i++) {
			const dk_flat_op *op = &ops[rem[i]];
			uint64_t sup = support(op);
			int ok = !(sup & blocked) && kinds[rem[i]] != 0 &&
				 nt < lim->max_gates &&
				 (lim->fuse || nt == 0);
			if (ok) {
				uint64_t nq = Q | target_mask(op);
				int me = mat_entries(kinds[rem[i]], op->k);
				if (popc(nq) <= m && nmat + me <= lim->max_mat) {
					Q = nq;
					take[nt++] = rem[i];
					nmat += me;
					continue;
				}
			}
			defer[nd++] = rem[i];
			blocked |= sup;
		}
		if (nt == 0) {
			/* cannot happen with the cap above; never emit an empty sweep */
			steps[nsteps].kind = 2;
			steps[nsteps].op_index = rem[0];
			steps[nsteps].ngates = 1;
			nsteps++;
			memmove(rem, rem + 1, sizeof(int) * (size_t)(nrem - 1));
			nrem--;
			continue;
		}
		/* complete Q to m bits with the lowest free qubits */
		for (unsigned q = 0; popc(Q) < m && q < n; q++)
			Q |= UINT64_C(1) << q;
		if (emit_sweep(&b, ops, take, nt, Q, n, prec, m, kinds,
			       &steps[nsteps]))
			goto fail;
		nsteps++;
		memcpy(rem, defer, sizeof(int) * (size_t)nd);
		nrem = nd;
	}
	plan->steps = steps;
	plan->nsteps = nsteps;
	plan->blob = b.p;
	plan->blob_bytes = b.len;
	free(rem);
	free(defer);
	free(take);
	free(kinds);
	return 0;
fail:
	free(rem);
	free(defer);
	free(take);
	free(kinds);
	free(steps);
	free(b.p);
	memset(plan, 0, sizeof(*plan));
	return DK_ERR_ALLOC;
}

void dk_plan_free(dk_plan *plan)
{
	free(plan->steps);
	free(plan->blob);
	memset(plan, 0, sizeof(*plan));
}
