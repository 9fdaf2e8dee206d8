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
	if (lim->tensor >= 0)
		m = DK_TILE_BITS_TC; /* tensor sweeps: 4 passes, two chained pairs */
	if (lim->tile_bits >= DK_PASS_BITS && lim->tile_bits <= 12)
		m = lim->tile_bits; /* caller's choice */
	if ((int)n < m)
		m = (int)n;
	lim->tile_bits = m;
	/* pinned low qubits: tensor sweeps pin 2 (contiguous runs of 64 bytes
	 * for complex128, 32 for complex64): the freer tile choice gives fewer
	 * sweeps (30 qubits, depth 40: 65 against 83), which outweighs the
	 * slower streaming of shorter runs at both precisions.  Scalar sweeps
	 * pin 4. */
	const int low = lim->tensor >= 0 ? 2 : 4;
	lim->low_bits = m < low ? m : low;
	lim->max_gates = 512;
	lim->max_passes = 512;
	lim->max_mat = 4096; /* complex entries: <= 64 KiB of a sweep's shared memory */
	lim->fuse = 1;
	lim->fold = lim->fold > 0 ? lim->fold : (lim->fold < 0 ? 0 : DK_FOLD_DEFAULT);
	lim->tensor = lim->tensor < 0 ? 0 : 1;
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

/* Per-pass address tables for an explicit thread-bit -> tile-bit map:
 * thread bit j (j < nl) carries tile bit lane[j]. */
static void pass_tables_lanes(dk_pass_desc *pd, const uint8_t *pb, const uint8_t *lane,
			      int nl, int sw)
{
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

static void pass_tables(dk_pass_desc *pd, const uint8_t *pb, int m, int sw)
{
	uint8_t lane[32];
	const int nl = lane_map(m, pb, sw, lane);
	pass_tables_lanes(pd, pb, lane, nl, sw);
}

/* Lane bits of the passes of a phase whose warp bits are W: every residue
 * mod `res` present among the lane bits of a pass makes its quarter-warp
 * (half-warp) accesses conflict free. */
static int phase_score(const uint32_t *pmask, int cnt, uint32_t W, int m, int res)
{
	/* a pass scores when its lane bits L meet every residue class mod res */
	uint32_t cls[8] = { 0 };
	for (int b = 0; b < m; b++)
		cls[b % res] |= 1u << b;
	int score = 0;
	for (int i = 0; i < cnt; i++) {
		const uint32_t L = ((1u << m) - 1u) & ~pmask[i] & ~W;
		int all = 1;
		for (int r = 0; r < res && all; r++)
			all = (L & cls[r]) != 0;
		score += all;
	}
	return score;
}

/* Tensor sweeps read and write a pass's columns in two patterns: a gather
 * whose quarter-warp (16-byte amplitudes) or half-warp (8-byte) varies thread
 * bit 0 (and 1 for 8-byte) with pass bits 0 and 1, and a scatter that varies
 * pass bit 0 (and 1) with thread bits 1 and 2.  Under the XOR swizzle each
 * tile bit b moves the bank group by the unit vector of b mod res, so a phase
 * takes 2^(varying bits - distinct residues) wavefronts. */
static int nres(const int *b, int cnt, int res)
{
	unsigned seen = 0;
	for (int i = 0; i < cnt; i++)
		seen |= 1u << (b[i] % res);
	return popc(seen);
}

/* Wavefronts of a pass's gather and scatter per quarter-warp group, from the
 * bank groups (bit % res) of pass bits 0, 1 and thread bits 0..2. */
static int tc_cost(int pb0, int pb1, int l0, int l1, int l2, int res)
{
	if (res == 3) {
		const int g = popc((1u << l0) | (1u << pb0) | (1u << pb1));
		const int t = popc((1u << pb0) | (1u << l1) | (1u << l2));
		return (1 << (3 - g)) + (1 << (3 - t));
	}
	const int g = popc((1u << l0) | (1u << l1) | (1u << pb0) | (1u << pb1));
	const int t = popc((1u << pb0) | (1u << pb1) | (1u << l1) | (1u << l2));
	return (1 << (4 - g)) + (1 << (4 - t));
}

/* Cheapest order of pass bits P (register bits 0..2) and choice of thread
 * bits 0..2 among the lane bits L; returns the cost. */
static int tc_best(uint32_t P, uint32_t L, int m, int res, uint8_t *pb, uint8_t *l3)
{
	int p[DK_PASS_BITS], np = 0, l[32], nl = 0, best = 1 << 30;
	int pr[DK_PASS_BITS], lr[32]; /* their bank groups */
	for (int b = 0; b < m; b++) {
		if (P >> b & 1u) {
			pr[np] = b % res;
			p[np++] = b;
		} else if (L >> b & 1u) {
			lr[nl] = b % res;
			l[nl++] = b;
		}
	}
	static const int perm[6][3] = { { 0, 1, 2 }, { 0, 2, 1 }, { 1, 0, 2 },
					{ 1, 2, 0 }, { 2, 0, 1 }, { 2, 1, 0 } };
	for (int o = 0; o < 6; o++)
		for (int a = 0; a < nl; a++)
			for (int b2 = 0; b2 < nl; b2++)
				for (int c = 0; c < nl; c++) {
					if (a == b2 || a == c || b2 == c)
						continue;
					const int cost = tc_cost(pr[perm[o][0]], pr[perm[o][1]], lr[a],
								 lr[b2], lr[c], res);
					if (cost < best) {
						best = cost;
						if (pb)
							for (int j = 0; j < 3; j++)
								pb[j] = (uint8_t)p[perm[o][j]];
						if (l3) {
							l3[0] = (uint8_t)l[a];
							l3[1] = (uint8_t)l[b2];
							l3[2] = (uint8_t)l[c];
						}
					}
				}
	return best;
}

/* The cost tc_best returns, without the choice: tc_cost depends on the lane
 * bits only through their bank groups (bit % res), so the search runs over
 * groups, each used at most as often as L has bits in it -- the same
 * minimum over res^3 group triples instead of every ordered bit triple. */
static int tc_best_cost(uint32_t P, uint32_t L, int m, int res)
{
	int p[DK_PASS_BITS], np = 0, cnt[4] = { 0, 0, 0, 0 }, best = 1 << 30;
	for (int b = 0; b < m; b++) {
		if (P >> b & 1u)
			p[np++] = b % res;
		else if (L >> b & 1u)
			cnt[b % res]++;
	}
	static const int perm[6][3] = { { 0, 1, 2 }, { 0, 2, 1 }, { 1, 0, 2 },
					{ 1, 2, 0 }, { 2, 0, 1 }, { 2, 1, 0 } };
	for (int o = 0; o < 6; o++)
		for (int x = 0; x < res; x++) {
			if (cnt[x] < 1)
				continue;
			for (int y = 0; y < res; y++) {
				if (cnt[y] < 1 + (y == x))
					continue;
				for (int z = 0; z < res; z++) {
					if (cnt[z] < 1 + (z == x) + (z == y))
						continue;
					const int cost = tc_cost(p[perm[o][0]], p[perm[o][1]], x, y, z,
								 res);
					if (cost < best)
						best = cost;
				}
			}
		}
	return best;
}

/* What build_phase needs to know about the gates of a sweep (tensor
 * sweeps) to decide which pairs of passes can chain in registers. */
typedef struct phase_ctx {
	const dk_flat_op *ops;
	const int *order; /* gates of the sweep in pass order */
	const int8_t *loc_of; /* tile bit of each qubit, -1 outside the tile */
	unsigned n;
} phase_ctx;

static int tc_local(const dk_flat_op *op, const int8_t *loc_of, const uint32_t *preg);
static void tile_cond(const dk_flat_op *op, const int8_t *loc_of, unsigned n, uint64_t *gc,
		      uint64_t *ga);

/* A pass of a tensor sweep folds into exactly one gate-list entry when all
 * its gates are pass-local and carry at most DK_VAR_MAX distinct tile
 * conditions. */
static int single_entry(const phase_ctx *cx, const dk_pass_desc *pd, uint32_t P)
{
	if (pd->g1 <= pd->g0)
		return 0;
	uint32_t preg[64];
	memset(preg, 0xff, sizeof(preg));
	int r = 0;
	for (int b = 0; b < 32; b++)
		if (P >> b & 1u)
			preg[b] = (uint32_t)r++;
	uint64_t cgc[DK_VAR_MAX], cga[DK_VAR_MAX];
	int nv = 0;
	for (int g = pd->g0; g < pd->g1; g++) {
		const dk_flat_op *op = &cx->ops[cx->order[g]];
		if (!tc_local(op, cx->loc_of, preg))
			return 0;
		uint64_t gc, ga;
		tile_cond(op, cx->loc_of, cx->n, &gc, &ga);
		if (!(gc | ga))
			continue;
		int j = 0;
		while (j < nv && (cgc[j] != gc || cga[j] != ga))
			j++;
		if (j == nv) {
			if (nv == DK_VAR_MAX)
				return 0;
			cgc[nv] = gc;
			cga[nv] = ga;
			nv++;
		}
	}
	return 1;
}

static const int perm3[6][3] = { { 0, 1, 2 }, { 0, 2, 1 }, { 1, 0, 2 },
				 { 1, 2, 0 }, { 2, 0, 1 }, { 2, 1, 0 } };

/* Fewest shared-memory wavefronts of a chained pair's gather (pass A) and
 * scatter (pass B) over the orders of A's bits a and B's bits c (each in
 * increasing order, permuted by perm3[*bo] and perm3[*bp]). */
static int chain_orders(uint32_t PA, uint32_t PB, int m, int res, int *bo, int *bp)
{
	int a[3], c[3], na = 0, nc = 0;
	for (int b = 0; b < m; b++) {
		if (PA >> b & 1u)
			a[na++] = b;
		else if (PB >> b & 1u)
			c[nc++] = b;
	}
	int best = 1 << 30;
	*bo = *bp = 0;
	for (int o = 0; o < 6; o++)
		for (int q = 0; q < 6; q++) {
			const int a0 = a[perm3[o][0]], a1 = a[perm3[o][1]], a2 = a[perm3[o][2]];
			const int c0 = c[perm3[q][0]], c1 = c[perm3[q][1]], c2 = c[perm3[q][2]];
			int cost;
			if (res == 3) {
				const int g[3] = { c0, a0, a1 }, t[3] = { c1, a1, a2 };
				cost = (1 << (3 - nres(g, 3, 3))) + (1 << (3 - nres(t, 3, 3)));
			} else {
				const int g[4] = { c0, c1, a0, a1 }, t[4] = { c1, c2, a1, a2 };
				cost = (1 << (4 - nres(g, 4, res))) + (1 << (4 - nres(t, 4, res)));
			}
			if (cost < best) {
				best = cost;
				*bo = o;
				*bp = q;
			}
		}
	return best;
}

/* Lane tables of a chained pair: pass A (bits a0 a1 a2, thread bits c0 c1
 * c2 r0 r1 W...) and pass B = (c1 c2 c0, thread bits a0 a1 a2 r0 r1 W...),
 * the orders picked for the fewest shared-memory wavefronts of A's gather
 * and B's scatter. */
static void chain_pair(dk_pass_desc *pa, dk_pass_desc *pb, uint32_t PA, uint32_t PB, uint32_t W,
		       int m, int res, uint8_t *pbA, uint8_t *pbB)
{
	int a[3], c[3], r[2], na = 0, nc = 0, nr = 0;
	for (int b = 0; b < m; b++) {
		if (PA >> b & 1u)
			a[na++] = b;
		else if (PB >> b & 1u)
			c[nc++] = b;
		else if (!(W >> b & 1u) && nr < 2)
			r[nr++] = b;
	}
	const int(*perm)[3] = perm3;
	int bo, bp;
	chain_orders(PA, PB, m, res, &bo, &bp);
	uint8_t laneA[32], laneB[32];
	int nl = 0;
	for (int j = 0; j < 3; j++) {
		pbA[j] = (uint8_t)a[perm[bo][j]];
		laneA[j] = (uint8_t)c[perm[bp][j]];
		laneB[j] = pbA[j];
	}
	pbB[0] = laneA[1];
	pbB[1] = laneA[2];
	pbB[2] = laneA[0];
	nl = 3;
	for (int j = 0; j < nr; j++, nl++)
		laneA[nl] = laneB[nl] = (uint8_t)r[j];
	for (int b = 0; b < m; b++)
		if (W >> b & 1u) {
			laneA[nl] = laneB[nl] = (uint8_t)b;
			nl++;
		}
	pass_tables_lanes(pa, pbA, laneA, nl, res);
	pass_tables_lanes(pb, pbB, laneB, nl, res);
}

/* Bits of a chained pair: A and B (disjoint target bits) each filled up to
 * DK_PASS_BITS bits with disjoint fillers, chosen for the fewest
 * shared-memory wavefronts of the pair (chain_orders), then for the fewest
 * bits outside the phase's bits F (which may grow to fmax bits), then for
 * the highest bits, as the plain fill takes them.  F holds at least
 * 2 * DK_PASS_BITS bits, so a choice inside it always exists. */
static void fill_pair(uint32_t A, uint32_t B, uint32_t F, int fmax, int m, int res,
		      uint32_t *PA, uint32_t *PB)
{
	const uint32_t pool = ((1u << m) - 1u) & ~(A | B);
	const int na = DK_PASS_BITS - popc(A), nb = DK_PASS_BITS - popc(B);
	int best = 1 << 30;
	*PA = A;
	*PB = B;
	/* submasks in decreasing order: the first of each size has the
	 * highest bits */
	for (uint32_t x = pool;; x = (x - 1) & pool) {
		if (popc(x) == na) {
			const uint32_t rest = pool & ~x;
			for (uint32_t y = rest;; y = (y - 1) & rest) {
				if (popc(y) == nb && popc(F | x | y) <= fmax) {
					int bo, bp;
					/* wavefronts first, then bits outside F */
					const int c = 64 * chain_orders(A | x, B | y, m, res, &bo, &bp) +
						      popc((x | y) & ~F);
					if (c < best) {
						best = c;
						*PA = A | x;
						*PB = B | y;
					}
				}
				if (y == 0)
					break;
			}
		}
		if (x == 0)
			break;
	}
}

/* A phase: consecutive passes [0, cnt) whose pass bits all avoid the same
 * `wbits` tile bits W, which every pass maps to the thread bits above the 5
 * lane bits.  A warp then touches the same tile slots in every pass of the
 * phase, so consecutive passes only need a warp barrier.  `need[i]` are the
 * target bits of pass i; they are filled up to DK_PASS_BITS from the phase's
 * union first (keeping it small), W is picked from the rest.
 *
 * Tensor sweeps: two neighbouring single-entry passes whose target bits are
 * disjoint chain in registers when their filled bit sets are disjoint too.
 * Such pairs are marked first (greedily from the front, which gives the most
 * pairs on a path) and filled from disjoint bits (fill_pair); the phase's
 * union grows to at least 2 * DK_PASS_BITS and at most m - wbits bits, which
 * still leaves the wbits warp bits and the 2 lane bits a chained pair maps
 * besides its 6 pass bits (m - wbits = DK_PASS_BITS + 5). */
static void build_phase(dk_pass_desc *pd, const uint32_t *need, int cnt, int m, int wbits,
			int res, int tensor, const phase_ctx *cx,
			uint8_t (*pbits)[DK_PASS_BITS])
{
	uint32_t F = 0, pmask[64];
	uint8_t pair[64] = { 0 }; /* pass i chains with pass i + 1 */
	for (int i = 0; i < cnt; i++)
		F |= need[i];
	for (int bit = m - 1; popc(F) < DK_PASS_BITS && bit >= 0; bit--)
		F |= 1u << bit;
	if (tensor && cx && wbits >= 0 && m - wbits >= 2 * DK_PASS_BITS) {
		for (int i = 0; i + 1 < cnt; i++) {
			if ((need[i] & need[i + 1]) || !single_entry(cx, &pd[i], need[i]) ||
			    !single_entry(cx, &pd[i + 1], need[i + 1]))
				continue;
			for (int bit = m - 1; popc(F) < 2 * DK_PASS_BITS && bit >= 0; bit--)
				F |= 1u << bit;
			pair[i] = 1;
			i++;
		}
	}
	for (int i = 0; i < cnt; i++) {
		uint32_t P = need[i];
		if (pair[i]) {
			fill_pair(need[i], need[i + 1], F, m - wbits, m, res, &P, &pmask[i + 1]);
			F |= P | pmask[i + 1];
		} else if (i > 0 && pair[i - 1]) {
			P = pmask[i]; /* filled with its partner */
		}
		for (int bit = m - 1; popc(P) < DK_PASS_BITS && bit >= 0; bit--)
			if (F & (1u << bit))
				P |= 1u << bit;
		pmask[i] = P;
		int j = 0;
		for (int bit = 0; bit < m; bit++)
			if (P & (1u << bit))
				pbits[i][j++] = (uint8_t)bit;
	}
	/* warp bits: the subset of the free bits that keeps the most passes
	 * conflict free (first one found on ties) */
	const uint32_t pool = ((1u << m) - 1u) & ~F;
	uint32_t W = 0;
	int best = 0, have = 0;
	for (uint32_t x = pool;; x = (x - 1) & pool) {
		if (popc(x) == wbits) {
			int sc;
			if (tensor) {
				/* fewest shared-memory wavefronts of the tensor passes */
				sc = 0;
				for (int i = 0; i < cnt; i++)
					sc -= tc_best_cost(pmask[i], ((1u << m) - 1u) & ~pmask[i] & ~x, m,
							   res);
			} else {
				sc = phase_score(pmask, cnt, x, m, res);
			}
			if (!have || sc > best) {
				best = sc;
				W = x;
				have = 1;
			}
		}
		if (x == 0)
			break;
	}
	if (tensor) {
		for (int i = 0; i < cnt; i++) {
			/* a pair of single-entry passes on disjoint bits chains
			 * (never one that would split a pair marked above) */
			if (cx && wbits >= 0 && i + 1 < cnt && !(pmask[i] & pmask[i + 1]) &&
			    (pair[i] || !pair[i + 1]) &&
			    single_entry(cx, &pd[i], pmask[i]) &&
			    single_entry(cx, &pd[i + 1], pmask[i + 1])) {
				chain_pair(&pd[i], &pd[i + 1], pmask[i], pmask[i + 1], W, m, res,
					   pbits[i], pbits[i + 1]);
				pd[i].flags |= DK_PASS_WARP | DK_PASS_CHAIN;
				if (i + 2 < cnt)
					pd[i + 1].flags |= DK_PASS_WARP;
				i++;
				continue;
			}
			uint8_t lane[32], l3[3];
			const uint32_t L = ((1u << m) - 1u) & ~pmask[i] & ~W;
			tc_best(pmask[i], L, m, res, pbits[i], l3);
			int nl = 0;
			for (int j = 0; j < 3; j++)
				lane[nl++] = l3[j];
			for (int b = 0; b < m; b++)
				if ((L >> b & 1u) && b != l3[0] && b != l3[1] && b != l3[2])
					lane[nl++] = (uint8_t)b;
			for (int b = 0; b < m; b++)
				if (W & (1u << b))
					lane[nl++] = (uint8_t)b;
			pass_tables_lanes(&pd[i], pbits[i], lane, nl, res);
			if (i + 1 < cnt)
				pd[i].flags |= DK_PASS_WARP;
		}
		return;
	}
	for (int i = 0; i < cnt; i++) {
		uint8_t lane[32], free_bits[32];
		int nf = 0, nl = 0, taken[32] = { 0 };
		const uint32_t L = ((1u << m) - 1u) & ~pmask[i] & ~W;
		for (int b = 0; b < m; b++)
			if (L & (1u << b))
				free_bits[nf++] = (uint8_t)b;
		for (int r = 0; r < res; r++)
			for (int k = 0; k < nf; k++)
				if (!taken[k] && free_bits[k] % res == r) {
					lane[nl++] = free_bits[k];
					taken[k] = 1;
					break;
				}
		for (int k = 0; k < nf; k++)
			if (!taken[k])
				lane[nl++] = free_bits[k];
		for (int b = 0; b < m; b++)
			if (W & (1u << b))
				lane[nl++] = (uint8_t)b;
		pass_tables_lanes(&pd[i], pbits[i], lane, nl, res);
		if (i + 1 < cnt)
			pd[i].flags |= DK_PASS_WARP;
	}
}

/* ---- pass folding ------------------------------------------------------ */

typedef struct fold_params {
	int dispatch; /* cost of one gate on its own (0: no folding) */
	int max_mat; /* complex matrix entries of a sweep */
	int tensor; /* every gate list entry is an 8x8 product (tensor sweep) */
	int bank_mode; /* dk_plan_limits.bank_mode */
} fold_params;

/* ---- bank map of a tensor sweep --------------------------------------------
 * Under the layout of dk_sweep_hdr.bankv, tile bit b moves an access to bank
 * group v_b (e_b for the SW low bits).  A quarter-warp of 16-byte accesses
 * (half-warp of 8-byte ones) whose lanes vary the tile bits B takes
 * 2^(SW - rank{v_b : b in B}) wavefronts.  The planner fixes each pass's bit
 * orders first (with the residue model v_b = e_(b mod SW)), then picks the
 * v_b of the bits above SW that minimise the wavefronts of the accesses the
 * sweep's kernel makes, and derives the slot tables from the raw ones. */

typedef struct bank_pat {
	int w; /* accesses of this shape per tile */
	int nb;
	uint8_t b[4]; /* tile bits varied by the lanes of one wavefront group */
} bank_pat;

static int gf2_rank(const unsigned *v, int k)
{
	unsigned basis[4];
	int r = 0;
	for (int i = 0; i < k; i++) {
		unsigned x = v[i];
		for (int j = 0; j < r; j++)
			if ((x ^ basis[j]) < x)
				x ^= basis[j];
		if (x) {
			/* keep the basis reduced on its leading bits */
			basis[r++] = x;
			for (int a = r - 1; a > 0 && basis[a] > basis[a - 1]; a--) {
				const unsigned t = basis[a];
				basis[a] = basis[a - 1];
				basis[a - 1] = t;
			}
		}
	}
	return r;
}

static int pat_cost(const bank_pat *p, const unsigned *F, int sw)
{
	unsigned v[4];
	for (int i = 0; i < p->nb; i++)
		v[i] = F[p->b[i]];
	return p->w << (sw - gf2_rank(v, p->nb));
}

static int tile_bit(uint32_t mask) { return mask ? __builtin_ctz(mask) : 0; }

/* The wavefront-group shapes of a tensor sweep's passes.  mode 0 (mma.sync
 * kernels): a pass gathers with lanes on (thread bit 0 [, thread bit 1 for
 * 8-byte amplitudes], pass bits 0, 1) and scatters with lanes on (pass bit
 * 0 [, pass bit 1], thread bits 1, 2), twice per column group; a chained
 * pair gathers with its first pass and scatters with its second.  mode 1
 * (whole columns per thread): lanes on thread bits 0 .. SW-1, eight reads
 * and eight writes per column and entry. */
static int bank_patterns(const dk_pass_desc *pd, int npass, int sw, int mode, bank_pat *out)
{
	int np = 0;
	for (int i = 0; i < npass; i++) {
		const dk_pass_desc *a = &pd[i];
		const int chained = mode == 0 && (a->flags & DK_PASS_CHAIN) && i + 1 < npass;
		const dk_pass_desc *c = chained ? &pd[i + 1] : a;
		const int nent = chained ? 1 : (a->g1 > a->g0 ? a->g1 - a->g0 : 1);
		if (mode == 1) {
			bank_pat *p = &out[np++];
			p->w = 16 * nent;
			p->nb = sw;
			for (int j = 0; j < sw; j++)
				p->b[j] = (uint8_t)tile_bit(a->rlo[1u << j]);
			continue;
		}
		bank_pat *g = &out[np++], *t = &out[np++];
		g->w = t->w = 2 * nent;
		g->nb = t->nb = sw == 3 ? 3 : 4;
		if (sw == 3) {
			g->b[0] = (uint8_t)tile_bit(a->rlo[1]);
			g->b[1] = (uint8_t)tile_bit(a->pm[0]);
			g->b[2] = (uint8_t)tile_bit(a->pm[1]);
			t->b[0] = (uint8_t)tile_bit(c->pm[0]);
			t->b[1] = (uint8_t)tile_bit(c->rlo[2]);
			t->b[2] = (uint8_t)tile_bit(c->rlo[4]);
		} else {
			g->b[0] = (uint8_t)tile_bit(a->rlo[1]);
			g->b[1] = (uint8_t)tile_bit(a->rlo[2]);
			g->b[2] = (uint8_t)tile_bit(a->pm[0]);
			g->b[3] = (uint8_t)tile_bit(a->pm[1]);
			t->b[0] = (uint8_t)tile_bit(c->pm[0]);
			t->b[1] = (uint8_t)tile_bit(c->pm[1]);
			t->b[2] = (uint8_t)tile_bit(c->rlo[2]);
			t->b[3] = (uint8_t)tile_bit(c->rlo[4]);
		}
		if (chained)
			i++;
	}
	return np;
}

/* Local search for the v_b (b >= sw) of a tile of m bits, starting from the
 * residue map and from a few fixed pseudo-random maps; the cheapest wins
 * (the residue map on ties).  F: m entries, F[b] = e_b for b < sw. */
static void choose_bank_map(const bank_pat *pat, int np, int m, int sw, unsigned *F)
{
	const unsigned nv = 1u << sw;
	unsigned best[16], cur[16];
	for (int b = 0; b < m; b++)
		best[b] = b < sw ? 1u << b : 1u << (b % sw);
	int best_cost = 0;
	for (int i = 0; i < np; i++)
		best_cost += pat_cost(&pat[i], best, sw);
	int ideal = 0;
	for (int i = 0; i < np; i++)
		ideal += pat[i].w;
	uint32_t rng = 0x9e3779b9u;
	for (int start = 0; start < 4 && best_cost > ideal; start++) {
		for (int b = 0; b < m; b++) {
			if (b < sw || start == 0) {
				cur[b] = best[b];
			} else {
				rng = rng * 1664525u + 1013904223u;
				cur[b] = 1u + (rng >> 8) % (nv - 1u);
			}
		}
		int cost = 0;
		for (int i = 0; i < np; i++)
			cost += pat_cost(&pat[i], cur, sw);
		for (int improved = 1; improved && cost > ideal;) {
			improved = 0;
			for (int b = sw; b < m; b++) {
				/* cost of the patterns that use bit b, for each candidate */
				int base = 0;
				for (int i = 0; i < np; i++)
					for (int j = 0; j < pat[i].nb; j++)
						if (pat[i].b[j] == b) {
							base += pat_cost(&pat[i], cur, sw);
							break;
						}
				const unsigned keep = cur[b];
				unsigned pick = keep;
				int pick_cost = base;
				for (unsigned v = 1; v < nv; v++) {
					if (v == keep)
						continue;
					cur[b] = v;
					int c = 0;
					for (int i = 0; i < np; i++)
						for (int j = 0; j < pat[i].nb; j++)
							if (pat[i].b[j] == b) {
								c += pat_cost(&pat[i], cur, sw);
								break;
							}
					if (c < pick_cost) {
						pick_cost = c;
						pick = v;
					}
				}
				cur[b] = pick;
				if (pick != keep) {
					cost += pick_cost - base;
					improved = 1;
				}
			}
		}
		if (cost < best_cost) {
			best_cost = cost;
			memcpy(best, cur, sizeof(unsigned) * (size_t)m);
		}
	}
	memcpy(F, best, sizeof(unsigned) * (size_t)m);
}

static uint32_t swizzle_map(uint32_t i, const unsigned *F, int m, int sw)
{
	uint32_t f = 0;
	for (int b = sw; b < m; b++)
		if ((i >> b) & 1u)
			f ^= F[b];
	return i ^ f;
}

/* Slot tables of every pass from its raw tables under the map F, and the
 * map packed for the sweep header. */
static uint64_t apply_bank_map(dk_pass_desc *pd, int npass, const unsigned *F, int m, int sw)
{
	for (int i = 0; i < npass; i++) {
		dk_pass_desc *p = &pd[i];
		for (int j = 0; j < DK_PASS_BITS; j++)
			p->sp[j] = swizzle_map(p->pm[j], F, m, sw);
		for (int x = 0; x < 32; x++)
			p->slo[x] = swizzle_map(p->rlo[x], F, m, sw);
		for (int y = 0; y < 16; y++)
			p->shi[y] = swizzle_map(p->rhi[y], F, m, sw);
	}
	uint64_t packed = 0;
	for (int b = sw; b < m; b++)
		packed |= (uint64_t)(F[b] & 15u) << (4 * b);
	return packed;
}

/* The fixed XOR swizzle of scalar sweeps as a bank map (v_b = e_(b mod sw)). */
static uint64_t default_bank_map(int m, int sw)
{
	uint64_t packed = 0;
	for (int b = sw; b < m; b++)
		packed |= (uint64_t)(1u << (b % sw)) << (4 * b);
	return packed;
}

/* An entry of a sweep's gate list: a source gate (op >= 0) or a folded run
 * (op < 0); m8 is the 8x8 matrix in register order for DK_GK_DENSE3. */
typedef struct item_t {
	int op, kind, pass;
	int m8; /* first 8x8 matrix (register order) in the matrix buffer, -1: none */
	int nmat; /* matrices: 1, or 2^nvar for a variant entry */
	int nvar; /* variant entry: tile conditions cgc/cga[0..nvar) select the matrix */
	int has_cond; /* plain entry applied where cgc/cga[0] holds */
	uint64_t cgc[DK_VAR_MAX], cga[DK_VAR_MAX];
} item_t;

/* growable buffer of 8x8 complex matrices (128 doubles each) */
typedef struct mbuf_t {
	double *p;
	int n, cap;
} mbuf_t;

static int mbuf_add(mbuf_t *mb, int count)
{
	if (mb->n + count > mb->cap) {
		int nc = mb->cap ? mb->cap : 64;
		while (nc < mb->n + count)
			nc *= 2;
		double *np = (double *)realloc(mb->p, sizeof(double) * 128 * (size_t)nc);
		if (!np)
			return -1;
		mb->p = np;
		mb->cap = nc;
	}
	const int at = mb->n;
	mb->n += count;
	return at;
}

/* Tensor sweeps: a gate folds into a pass matrix when its targets and its
 * in-tile controls are pass bits; controls outside the tile become tile
 * conditions (matrix variants). */
static int tc_local(const dk_flat_op *op, const int8_t *loc_of, const uint32_t *preg)
{
	for (unsigned t = 0; t < op->k; t++) {
		const int lb = loc_of[op->tg[t]];
		if (lb < 0 || preg[lb] == 0xffffffffu)
			return 0;
	}
	const uint64_t c = op->cm | op->am;
	for (unsigned q = 0; q < 64; q++)
		if ((c >> q & 1u) && loc_of[q] >= 0 && preg[loc_of[q]] == 0xffffffffu)
			return 0;
	return 1;
}

static void tile_cond(const dk_flat_op *op, const int8_t *loc_of, unsigned n, uint64_t *gc,
		      uint64_t *ga)
{
	*gc = *ga = 0;
	for (unsigned q = 0; q < n; q++) {
		if (loc_of[q] >= 0)
			continue;
		const uint64_t bit = UINT64_C(1) << q;
		if (op->cm & bit)
			*gc |= bit;
		if (op->am & bit)
			*ga |= bit;
	}
}

/* FP64 FMAs per thread (8 amplitudes) of one gate of each kind */
static int fold_cost(int kind)
{
	switch (kind) {
	case DK_GK_DENSE1: return 64;
	case DK_GK_DENSE2: return 128;
	case DK_GK_DENSE3: return 256;
	case DK_GK_DIAG1:
	case DK_GK_ANTI1:
	case DK_GK_DIAGK: return 32;
	case DK_GK_PHASE1: return 16;
	default: return 0; /* SWAP1, NEG1: moves and sign flips */
	}
}

/* A gate folds into the 8x8 matrix of a pass when its targets and all its
 * controls are bits of the pass (preg[tile bit] = register bit, or ~0). */
static int foldable(const dk_flat_op *op, const int8_t *loc_of, const uint32_t *preg)
{
	for (unsigned t = 0; t < op->k; t++) {
		const int lb = loc_of[op->tg[t]];
		if (lb < 0 || preg[lb] == 0xffffffffu)
			return 0;
	}
	for (uint64_t c = op->cm | op->am; c; c &= c - 1) {
		const int lb = loc_of[__builtin_ctzll(c)];
		if (lb < 0 || preg[lb] == 0xffffffffu)
			return 0;
	}
	return 1;
}

static void identity8(double *M)
{
	memset(M, 0, sizeof(double) * 128);
	for (int r = 0; r < 8; r++)
		M[2 * (8 * r + r)] = 1.0;
}

/* 8x8 matrix, in register order, of a gate on the pass's bits: entry (r, c)
 * is the gate's entry (row(r), row(c)) where r and c agree outside the target
 * bits and the controls on pass bits hold on c, the identity elsewhere.
 * row(x) gathers the target bits of x, targets[0] lowest.  Controls off the
 * pass bits are left to the gate descriptor. */
static void gate8(const dk_flat_op *op, const int8_t *loc_of, const uint32_t *preg, double *G)
{
	unsigned treg[DK_SWEEP_MAX_K], tmask = 0, cr = 0, ar = 0;
	for (unsigned t = 0; t < op->k; t++) {
		treg[t] = preg[loc_of[op->tg[t]]];
		tmask |= 1u << treg[t];
	}
	for (unsigned q = 0; q < 64; q++) {
		const uint64_t bit = UINT64_C(1) << q;
		if (!((op->cm | op->am) & bit) || loc_of[q] < 0 ||
		    preg[loc_of[q]] == 0xffffffffu)
			continue;
		if (op->cm & bit)
			cr |= 1u << preg[loc_of[q]];
		else
			ar |= 1u << preg[loc_of[q]];
	}
	const uint64_t d = op->gate->dim;
	const double *g = op->gate->m;
	memset(G, 0, sizeof(double) * 128);
	for (unsigned r = 0; r < 8; r++)
		for (unsigned c = 0; c < 8; c++) {
			if ((r & ~tmask) != (c & ~tmask))
				continue;
			double *e = G + 2 * (8 * r + c);
			if ((c & cr) != cr || (c & ar)) {
				e[0] = (r == c) ? 1.0 : 0.0;
				continue;
			}
			unsigned gr = 0, gcn = 0;
			for (unsigned t = 0; t < op->k; t++) {
				gr |= ((r >> treg[t]) & 1u) << t;
				gcn |= ((c >> treg[t]) & 1u) << t;
			}
			e[0] = g[2 * (gr * d + gcn)];
			e[1] = g[2 * (gr * d + gcn) + 1];
		}
}

/* M = G * M (8x8 complex, row-major, interleaved) */
static void mul8(const double *G, double *M)
{
	double T[128];
	for (int r = 0; r < 8; r++)
		for (int c = 0; c < 8; c++) {
			double re = 0.0, im = 0.0;
			for (int k = 0; k < 8; k++) {
				const double *a = G + 2 * (8 * r + k), *b = M + 2 * (8 * k + c);
				re += a[0] * b[0] - a[1] * b[1];
				im += a[0] * b[1] + a[1] * b[0];
			}
			T[2 * (8 * r + c)] = re;
			T[2 * (8 * r + c) + 1] = im;
		}
	memcpy(M, T, sizeof(T));
}

/* Emit one sweep program for ops[idx[0..cnt)] over tile set Q. */
static int emit_sweep(blob_t *b, const dk_flat_op *ops, const int *idx,
		      int cnt, uint64_t Q, unsigned n, int prec, int m,
		      const int *kinds, const fold_params *fold, dk_step *step)
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
	uint32_t *need = (uint32_t *)calloc((size_t)(cnt ? cnt : 1), sizeof(uint32_t));
	if (!rem || !defer || !order || !passes || !pbits || !need) {
		free(rem);
		free(defer);
		free(order);
		free(passes);
		free(pbits);
		free(need);
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
			if (fold->tensor) {
				/* tensor sweeps: keep a gate's in-tile controls in its
				 * pass when they fit, so the gate folds into the pass
				 * matrix instead of needing a product of its own */
				uint32_t sl = tl;
				for (unsigned q = 0; q < n; q++)
					if (((op->cm | op->am) >> q & 1u) && loc_of[q] >= 0)
						sl |= 1u << loc_of[q];
				if (popc(sl) <= DK_PASS_BITS)
					tl = sl;
			}
			if (popc(P | tl) <= DK_PASS_BITS) {
				P |= tl;
				order[nord++] = rem[i];
			} else {
				defer[nd++] = rem[i];
				blocked |= sup;
			}
		}
		pd->g1 = (uint16_t)nord;
		need[npass] = P;
		for (int g = pd->g0; g < pd->g1; g++) {
			const dk_flat_op *op = &ops[order[g]];
			if ((op->cm | op->am) & Q)
				pd->flags |= DK_PASS_CTL;
		}
		npass++;
		memcpy(rem, defer, sizeof(int) * (size_t)nd);
		nrem = nd;
	}

	/* Pass bits and lane tables.  With at least one full warp per tile
	 * (m >= 8) passes are grouped into warp phases: a run of passes whose
	 * target bits fit in m - wbits tile bits (wbits = thread bits above the
	 * lanes).  Narrower tiles fill each pass with the highest free bits. */
	const int wbits = m - DK_PASS_BITS - 5;
	const phase_ctx cx = { ops, order, loc_of, n };
	/* tensor sweeps: neighbouring passes that can chain (disjoint target
	 * bits, one entry each), marked greedily from the front as build_phase
	 * does; a phase is cut before such a pair rather than between its two
	 * passes, trading a block barrier for a chained pair */
	uint8_t *pairs = (uint8_t *)calloc((size_t)(npass ? npass : 1), 1);
	if (!pairs) {
		free(rem);
		free(defer);
		free(order);
		free(passes);
		free(pbits);
		free(need);
		return -1;
	}
	if (fold->tensor && wbits >= 0 && m - wbits >= 2 * DK_PASS_BITS)
		for (int i = 0; i + 1 < npass; i++)
			if (!(need[i] & need[i + 1]) && single_entry(&cx, &passes[i], need[i]) &&
			    single_entry(&cx, &passes[i + 1], need[i + 1])) {
				pairs[i] = 1;
				i++;
			}
	for (int p0 = 0; p0 < npass;) {
		int p1 = p0 + 1;
		if (wbits >= 0) {
			uint32_t U = need[p0];
			while (p1 < npass && p1 - p0 < 64 && popc(U | need[p1]) <= m - wbits)
				U |= need[p1++];
			if (p1 < npass && p1 - 1 > p0 && pairs[p1 - 1])
				p1--;
			build_phase(&passes[p0], &need[p0], p1 - p0, m, wbits, res, fold->tensor,
				    fold->tensor ? &cx : NULL, &pbits[p0]);
		} else {
			uint32_t P = need[p0];
			for (int bit = m - 1; popc(P) < DK_PASS_BITS && bit >= 0; bit--)
				P |= 1u << bit;
			int j = 0;
			for (int bit = 0; bit < m; bit++)
				if (P & (1u << bit))
					pbits[p0][j++] = (uint8_t)bit;
			pass_tables(&passes[p0], pbits[p0], m, res);
		}
		p0 = p1;
	}
	free(pairs);

	/* Gate-list entries.  Scalar sweeps: a run of consecutive gates of a
	 * pass that act only on the pass's bits (targets and controls) and on
	 * every tile is replaced by its 8x8 product when that is cheaper than
	 * applying the gates one by one; dense 3-qubit gates are stored in
	 * register order.  Tensor sweeps: every entry is 8x8; a run of gates
	 * whose targets and in-tile controls are pass bits becomes one entry,
	 * with one matrix per combination of the run's (at most DK_VAR_MAX)
	 * distinct conditions on qubits outside the tile. */
	item_t *items = (item_t *)calloc((size_t)(nord ? nord : 1), sizeof(item_t));
	mbuf_t mb = { NULL, 0, 0 };
	if (!items) {
		free(rem);
		free(defer);
		free(order);
		free(passes);
		free(pbits);
		free(need);
		return -1;
	}
	int nit = 0, tot_mat = 0, oom = 0;
	for (int i = 0; i < nord; i++)
		tot_mat += mat_entries(kinds[order[i]], ops[order[i]].k);
	for (int pi = 0; pi < npass && !oom; pi++) {
		const int g0 = passes[pi].g0, g1 = passes[pi].g1;
		uint32_t preg[64];
		memset(preg, 0xff, sizeof(preg));
		for (int r = 0; r < DK_PASS_BITS; r++)
			preg[pbits[pi][r]] = (uint32_t)r;
		passes[pi].g0 = (uint16_t)nit;
		for (int g = g0; g < g1 && !oom;) {
			item_t *it = &items[nit];
			memset(it, 0, sizeof(*it));
			it->pass = pi;
			it->m8 = -1;
			if (fold->tensor && tc_local(&ops[order[g]], loc_of, preg)) {
				int e = g, all_cond = 1;
				while (e < g1 && tc_local(&ops[order[e]], loc_of, preg)) {
					uint64_t gc, ga;
					tile_cond(&ops[order[e]], loc_of, n, &gc, &ga);
					if (gc | ga) {
						int j = 0;
						while (j < it->nvar && (it->cgc[j] != gc || it->cga[j] != ga))
							j++;
						if (j == it->nvar) {
							if (it->nvar == DK_VAR_MAX)
								break;
							it->cgc[j] = gc;
							it->cga[j] = ga;
							it->nvar++;
						}
					} else {
						all_cond = 0;
					}
					e++;
				}
				/* one condition shared by every gate of the run: a plain
				 * entry skipped by the other tiles (chained passes keep
				 * the identity as the other variant instead) */
				const int chained = (passes[pi].flags & DK_PASS_CHAIN) ||
						    (pi > 0 && (passes[pi - 1].flags & DK_PASS_CHAIN));
				if (it->nvar == 1 && all_cond && !chained) {
					it->nvar = 0;
					it->has_cond = 1;
				}
				it->op = -1;
				it->kind = DK_GK_DENSE3;
				it->nmat = 1 << it->nvar;
				it->m8 = mbuf_add(&mb, it->nmat);
				if (it->m8 < 0) {
					oom = 1;
					break;
				}
				for (int v = 0; v < it->nmat; v++) {
					double *M = mb.p + 128 * (size_t)(it->m8 + v);
					identity8(M);
					for (int j = g; j < e; j++) {
						uint64_t gc, ga;
						tile_cond(&ops[order[j]], loc_of, n, &gc, &ga);
						int on = 1;
						for (int c = 0; c < it->nvar; c++)
							if (it->cgc[c] == gc && it->cga[c] == ga)
								on = (v >> c) & 1;
						if (!on)
							continue;
						double G[128];
						gate8(&ops[order[j]], loc_of, preg, G);
						mul8(G, M);
					}
				}
				nit++;
				g = e;
				continue;
			}
			if (!fold->tensor) {
				int e = g, run_cost = 0, run_mat = 0;
				while (e < g1 && foldable(&ops[order[e]], loc_of, preg)) {
					run_cost += fold_cost(kinds[order[e]]) + fold->dispatch;
					run_mat += mat_entries(kinds[order[e]], ops[order[e]].k);
					e++;
				}
				const int fused_cost = fold_cost(DK_GK_DENSE3) + fold->dispatch;
				if (e - g >= 2 && fold->dispatch > 0 && run_cost > fused_cost &&
				    tot_mat - run_mat + 64 <= fold->max_mat) {
					it->op = -1;
					it->kind = DK_GK_DENSE3;
					it->nmat = 1;
					it->m8 = mbuf_add(&mb, 1);
					if (it->m8 < 0) {
						oom = 1;
						break;
					}
					double *M = mb.p + 128 * (size_t)it->m8;
					identity8(M);
					for (int j = g; j < e; j++) {
						double G[128];
						gate8(&ops[order[j]], loc_of, preg, G);
						mul8(G, M);
					}
					tot_mat += 64 - run_mat;
					nit++;
					g = e;
					continue;
				}
			}
			/* a single gate; 8x8 in register order when it is a dense
			 * 3-qubit gate or the sweep is a tensor sweep */
			it->op = order[g];
			it->kind = kinds[order[g]];
			if (it->kind == DK_GK_DENSE3 || fold->tensor) {
				it->kind = DK_GK_DENSE3;
				it->nmat = 1;
				it->m8 = mbuf_add(&mb, 1);
				if (it->m8 < 0) {
					oom = 1;
					break;
				}
				gate8(&ops[order[g]], loc_of, preg, mb.p + 128 * (size_t)it->m8);
			}
			nit++;
			g++;
		}
		passes[pi].g1 = (uint16_t)nit;
		/* a chained pair needs exactly one entry in each pass */
		if (pi > 0 && (passes[pi - 1].flags & DK_PASS_CHAIN) &&
		    (passes[pi - 1].g1 - passes[pi - 1].g0 != 1 || passes[pi].g1 - passes[pi].g0 != 1))
			passes[pi - 1].flags &= ~(uint32_t)DK_PASS_CHAIN;
		/* controls inside the tile, after folding */
		passes[pi].flags &= ~(uint32_t)DK_PASS_CTL;
		for (int k = passes[pi].g0; k < nit; k++) {
			const dk_flat_op *op = items[k].op >= 0 ? &ops[items[k].op] : NULL;
			if (op && ((op->cm | op->am) & Q))
				passes[pi].flags |= DK_PASS_CTL;
		}
	}

	/* size the program */
	int nmat = 0, ncond = 0;
	for (int i = 0; i < nit; i++) {
		nmat += items[i].m8 >= 0 ? 64 * items[i].nmat
					 : mat_entries(items[i].kind, ops[items[i].op].k);
		ncond += items[i].nvar + items[i].has_cond;
		if (items[i].op >= 0 && ((ops[items[i].op].cm | ops[items[i].op].am) & ~Q))
			ncond++;
	}
	size_t pass_off = align_up(sizeof(dk_sweep_hdr), 16);
	size_t gate_off = align_up(pass_off + sizeof(dk_pass_desc) * (size_t)npass, 16);
	size_t cond_off = align_up(gate_off + sizeof(dk_gate_desc) * (size_t)nit, 16);
	size_t mat_off = align_up(cond_off + sizeof(dk_gate_cond) * (size_t)ncond, 16);
	size_t bytes = align_up(mat_off + 16 * (size_t)nmat, 16);

	size_t start = align_up(b->len, 16);
	if (oom || blob_reserve(b, (start - b->len) + bytes)) {
		free(items);
		free(mb.p);
		free(rem);
		free(defer);
		free(order);
		free(passes);
		free(pbits);
		free(need);
		return -1;
	}
	memset(b->p + b->len, 0, (start - b->len) + bytes);
	b->len = start;
	unsigned char *base = b->p + start;
	dk_sweep_hdr *h = (dk_sweep_hdr *)base;
	h->m = m;
	h->n = (int32_t)n;
	h->npass = npass;
	h->ngate = nit;
	h->ntiles = UINT64_C(1) << (n - (unsigned)m);
	memcpy(h->qpos, qpos, (size_t)m);
	h->pass_off = (uint32_t)pass_off;
	h->gate_off = (uint32_t)gate_off;
	h->mat_off = (uint32_t)mat_off;
	h->bytes = (uint32_t)bytes;
	h->cond_off = (uint32_t)cond_off;
	h->ncond = (uint32_t)ncond;
	if (fold->tensor && npass > 0) {
		/* the bank map for the kernel that runs this sweep; the tcgen05
		 * complex64 kernel (whole columns) runs 12-bit tiles only */
		const int mode = (fold->bank_mode == 1 && prec == DK_C64 && m == 12) ? 1 : 0;
		bank_pat *pat = (bank_pat *)malloc(sizeof(bank_pat) * 2 * (size_t)npass);
		if (pat) {
			unsigned F[16];
			const int np = bank_patterns(passes, npass, res, mode, pat);
			choose_bank_map(pat, np, m, res, F);
			h->bankv = apply_bank_map(passes, npass, F, m, res);
			free(pat);
		} else {
			h->bankv = default_bank_map(m, res);
		}
	} else {
		h->bankv = default_bank_map(m, res);
	}
	memcpy(base + pass_off, passes, sizeof(dk_pass_desc) * (size_t)npass);

	dk_gate_desc *gd = (dk_gate_desc *)(base + gate_off);
	dk_gate_cond *conds = (dk_gate_cond *)(base + cond_off);
	double *mats = (double *)(base + mat_off);
	int moff = 0, all_touched = 0, ci = 0;
	for (int i = 0; i < nit; i++) {
		const int pi = items[i].pass;
		const int kind = items[i].kind;
		dk_gate_desc *g = &gd[i];
		/* tensor sweeps count matrix offsets in whole 8x8 matrices */
		g->mat = (uint16_t)(fold->tensor ? moff / 64 : moff);
		if (items[i].m8 >= 0) {
			/* 8x8 matrices in register order: fused runs, variants or a
			 * single gate whose controls on the pass bits are inside */
			uint64_t gc = 0, ga = 0;
			if (items[i].op >= 0) {
				const dk_flat_op *op = &ops[items[i].op];
				uint32_t pmask = 0;
				for (int r = 0; r < DK_PASS_BITS; r++)
					pmask |= 1u << pbits[pi][r];
				for (unsigned q = 0; q < n; q++) {
					uint64_t bit = UINT64_C(1) << q;
					if (loc_of[q] >= 0 && (pmask >> loc_of[q] & 1u))
						continue;
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
			} else if (items[i].has_cond) {
				gc = items[i].cgc[0];
				ga = items[i].cga[0];
			}
			if (gc == 0 && ga == 0) {
				all_touched = 1;
				g->gcond = 0xffff;
			} else {
				conds[ci].gc = gc;
				conds[ci].ga = ga;
				g->gcond = (uint16_t)ci++;
			}
			if (items[i].nvar > 0) {
				/* variant entry: lc packs the condition indices (10 bits
				 * each), la their count */
				g->lc = 0;
				for (int c = 0; c < items[i].nvar; c++) {
					conds[ci].gc = items[i].cgc[c];
					conds[ci].ga = items[i].cga[c];
					g->lc |= (uint32_t)ci++ << (10 * c);
				}
				g->la = (uint32_t)items[i].nvar;
				g->code = (uint16_t)DK_GC_DENSE3V;
			} else {
				g->code = (uint16_t)(DK_GC_DENSE3 + ((g->lc | g->la) != 0));
			}
			g->info = (uint16_t)(0 | (1 << 2) | (2 << 4) | (3u << 6) |
					     ((unsigned)DK_GK_DENSE3 << 8));
			memcpy(mats + 2 * moff, mb.p + 128 * (size_t)items[i].m8,
			       sizeof(double) * 128 * (size_t)items[i].nmat);
			moff += 64 * items[i].nmat;
			continue;
		}
		const dk_flat_op *op = &ops[items[i].op];
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
	h->mode = fold->tensor ? DK_SWEEP_TENSOR : DK_SWEEP_SCALAR;
	b->len = start + bytes;
	step->kind = 1;
	step->prog_off = start;
	step->op_index = -1;
	step->ngates = nord;
	free(items);
	free(mb.p);
	free(rem);
	free(defer);
	free(order);
	free(passes);
	free(pbits);
	free(need);
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
	/* tensor sweeps need a full warp of 8-amplitude columns per tile */
	const fold_params fold = { lim->fold > 0 ? lim->fold : 0, lim->max_mat,
				   lim->tensor > 0 && m >= DK_PASS_BITS + 5, lim->bank_mode };
	for (int i = 0; i < nops; i++) {
		rem[i] = i;
		kinds[i] = (ops[i].k <= DK_SWEEP_MAX_K && sweepable)
				   ? dk_gate_classify(ops[i].gate)
				   : 0;
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
		/* complete Q to m bits with the lowest free qubits.  One gate per
		 * sweep (no fusion): leave its controls and anticontrols out of the
		 * tile where the register has room, so that they become tile
		 * conditions and an in-place sweep skips the tiles where they fail
		 * (2 S 2^-c bytes moved for c such qubits instead of 2 S). */
		if (!lim->fuse && nt == 1) {
			const dk_flat_op *op = &ops[take[0]];
			const uint64_t cond = (op->cm | op->am) & ~Q;
			if ((unsigned)popc(cond) <= n - (unsigned)m)
				for (unsigned q = 0; popc(Q) < m && q < n; q++)
					if (!((cond >> q) & 1u))
						Q |= UINT64_C(1) << q;
		}
		for (unsigned q = 0; popc(Q) < m && q < n; q++)
			Q |= UINT64_C(1) << q;
		if (emit_sweep(&b, ops, take, nt, Q, n, prec, m, kinds, &fold,
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
