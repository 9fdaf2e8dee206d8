/*
 * Internal structures of the B200 state-vector engine (not part of the ABI).
 *
 * Host side: immutable logical registers (dk_state) over reference-counted
 * device buffers (dk_buf) with a persistent list of pending gates (dk_op).
 * Device side: one amplitude array + a small scalar block per buffer.
 */
#ifndef DK_INTERNAL_H_
#define DK_INTERNAL_H_

#include <stddef.h>
#include <stdint.h>

#include "dokigpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Largest gate the fused sweep executes in registers; larger gates go to the
 * generic kernel (any k <= DK_MAX_GATE_QUBITS). */
#define DK_SWEEP_MAX_K 3
#define DK_MAX_GATE_QUBITS 10

/* Per-buffer device scalars.  Logical amplitude = amp / norm.  csq is the
 * exact sum of |amp|^2 of the stored content (kept so that sweeps which skip
 * inactive tiles can still produce the reference's renormalisation). */
typedef struct dk_scal {
	double norm;
	double csq;
	double p_sel; /* last collapse: probability of the selected outcome */
	double pad;
	int32_t flag; /* last collapse: outcome (0/1) */
	int32_t zero_norm; /* set when a collapse produced norm 0 */
	int32_t pad2[2];
} dk_scal;

struct dk_gate {
	int refcount;
	unsigned k;
	uint64_t dim;
	double *m; /* host, 2 * dim * dim, row-major interleaved */
};

typedef struct dk_buf {
	int refcount; /* logical registers sharing this storage */
	unsigned n;
	int prec;
	void *d; /* amplitudes */
	size_t bytes;
	dk_scal *sc; /* device scalars */
} dk_buf;

typedef struct dk_op {
	int refcount;
	struct dk_op *prev; /* the op applied before this one (NULL = buffer) */
	struct dk_gate *gate;
	unsigned k;
	unsigned tg[DK_MAX_GATE_QUBITS];
	uint64_t cm, am;
	uint32_t depth; /* chain length including this op */
} dk_op;

struct dk_state {
	unsigned n;
	int prec;
	int slot; /* stream slot the register's work is queued on */
	int released;
	dk_buf *buf; /* NULL for 0-qubit registers */
	dk_op *pending; /* ops queued on top of buf's content */
	/* caches, valid while pending == NULL (a flushed register never changes) */
	int have_norm;
	double norm, csq;
	int have_marg;
	double *marg; /* n marginal sums S_q (raw content), host */
	int have_phase;
	double phase;
	double *hcache; /* logical amplitudes (complex128), small registers */
};

/* ---- fused sweep program (built on the host, read by the sweep kernel) -- */

#define DK_TILE_BITS_C128 11
#define DK_TILE_BITS_C64 11
#define DK_TILE_BITS_TC 12 /* tile bits of tensor-core sweeps */
#define DK_PASS_BITS 3
/* nibbles of a tile number (tile bits m >= 0, register <= 40 qubits) */
#define DK_DEP_NIBBLES 10
/* default pass-folding cost of one gate (FP64 FMAs per thread) */
#define DK_FOLD_DEFAULT 96

enum {
	DK_GK_DENSE1 = 1,
	DK_GK_DIAG1 = 2,
	DK_GK_ANTI1 = 3,
	DK_GK_DENSE2 = 4,
	DK_GK_DENSE3 = 5,
	DK_GK_DIAGK = 6,
	DK_GK_SWAP1 = 7, /* [[0,1],[1,0]]: exchange, no arithmetic */
	DK_GK_PHASE1 = 8, /* diag(1, d): scale the |1> half only */
	DK_GK_NEG1 = 9, /* diag(1, -1): negate the |1> half */
};

/* Gate descriptor of a sweep (16 bytes, one shared-memory load).  `code`
 * selects the kernel's specialised entry: for the one-qubit kinds it is
 * DK_GC_<KIND> + t0 + 3 * (has controls inside the tile); DK_GC_DENSE2 + the
 * index of the ordered register-bit pair; DK_GC_DIAGK.  `info` keeps the
 * kind (bits 8-11), k (6-7) and register bits t2 (4-5), t1 (2-3), t0 (0-1). */
typedef struct dk_gate_desc {
	uint16_t code;
	uint16_t mat; /* offset of the matrix in complex entries */
	uint16_t gcond; /* index into the global-condition table, 0xffff: none */
	uint16_t info;
	uint32_t lc, la; /* control / anticontrol masks over local (tile) bits */
} dk_gate_desc;

/* Controls outside the tile: the gate acts on a tile iff
 * (base & gc) == gc && !(base & ga) for the tile's base index. */
typedef struct dk_gate_cond {
	uint64_t gc, ga;
} dk_gate_cond;

enum {
	DK_GC_DENSE1 = 0,
	DK_GC_SWAP1 = 6,
	DK_GC_PHASE1 = 12,
	DK_GC_DIAG1 = 18,
	DK_GC_ANTI1 = 24,
	DK_GC_DENSE2 = 30, /* + pair index: (0,1) (0,2) (1,0) (1,2) (2,0) (2,1) */
	DK_GC_DIAGK = 36,
	DK_GC_NEG1 = 37,
	DK_GC_DENSE3 = 43, /* + 1 with controls inside the tile: 8x8 matrix in
			    * register order (a fused run or a 3-qubit gate) */
	DK_GC_DENSE3V = 45, /* tensor sweeps: 2^la matrices; lc packs la indices
			     * (10 bits each) of tile conditions; the tile uses
			     * matrix sum_j [condition j holds] 2^j */
};
/* most tile conditions of one variant entry */
#define DK_VAR_MAX 3

/* A pass: the gates [g0, g1) applied to the 8 amplitudes each thread
 * gathers from the shared tile.  The tile is stored under an XOR swizzle that
 * is linear over GF(2), so a thread's 8 slots are
 *   (slo[tid & 31] ^ shi[tid >> 5]) ^ (XOR of sp[j] over the set bits j of r),
 * and the raw tile index (for control predicates) is the same with rlo, rhi,
 * pm and OR.  The host precomputes these tables per pass. */
typedef struct dk_pass_desc {
	uint16_t g0, g1; /* gate range [g0, g1) */
	uint32_t flags; /* DK_PASS_CTL | DK_PASS_WARP */
	uint32_t sp[DK_PASS_BITS]; /* swizzled slot offset of pass bit j */
	uint32_t pm[DK_PASS_BITS]; /* raw tile-index mask of pass bit j */
	uint32_t slo[32], shi[16]; /* swizzled offsets of thread bits 0-4 / 5-8 */
	uint32_t rlo[32], rhi[16]; /* raw tile-index bits of the same */
} dk_pass_desc; /* 416 bytes */

enum {
	DK_PASS_CTL = 1u, /* a gate of the pass has controls inside the tile */
	DK_PASS_WARP = 2u, /* the next pass maps the same tile bits to the warp
			    * index: a warp barrier separates the two */
	DK_PASS_CHAIN = 4u, /* tensor sweeps: this pass and the next each hold one
			     * entry, and this pass's thread bits 0-2 are the next
			     * pass's bits in the order that makes this pass's MMA
			     * output the next pass's MMA input: the pair runs in
			     * registers between one gather and one scatter */
};

typedef struct dk_sweep_hdr {
	int32_t m; /* tile bits */
	int32_t n; /* register qubits */
	int32_t npass, ngate;
	int32_t all_touched; /* every tile has an unconditionally active gate */
	int32_t mode; /* DK_SWEEP_SCALAR or DK_SWEEP_TENSOR */
	uint64_t ntiles;
	uint8_t qpos[16]; /* global bit of local bit j (ascending) */
	uint32_t pass_off, gate_off, mat_off; /* byte offsets from the header */
	uint32_t bytes; /* total program bytes */
	uint32_t cond_off, ncond; /* global-condition table */
	/* Shared-memory layout of the tile: tile index i sits in slot
	 * i ^ (XOR over the set bits b of i of v_b), v_b = nibble b of bankv, a
	 * vector over the low SW bits of the slot (SW = 3 for 16-byte, 4 for
	 * 8-byte amplitudes; v_b = 0 for b < SW).  v_b is the bank-group
	 * direction of tile bit b.  Scalar sweeps use v_b = 2^(b mod SW) (the
	 * kernels' fixed XOR swizzle); tensor sweeps a map the planner picks for
	 * the sweep's own access patterns. */
	uint64_t bankv;
} dk_sweep_hdr;

/* Sweep execution modes.  SCALAR: the gate list holds any kinds, applied
 * by per-thread FP arithmetic on 8 register amplitudes.  TENSOR: every entry
 * is an 8x8 matrix in register order (controls on non-pass tile bits and
 * outside the tile in the descriptor), applied with FP64 tensor-core MMAs. */
enum { DK_SWEEP_SCALAR = 0, DK_SWEEP_TENSOR = 1 };

/* One step of a flush plan. */
typedef struct dk_step {
	int kind; /* 1 = fused sweep, 2 = generic single gate */
	size_t prog_off; /* sweep: offset of its program in the plan blob */
	int op_index; /* generic: index into the flat op array */
	int ngates;
} dk_step;

typedef struct dk_flat_op {
	const struct dk_gate *gate;
	unsigned k;
	unsigned tg[DK_MAX_GATE_QUBITS];
	uint64_t cm, am;
} dk_flat_op;

typedef struct dk_plan {
	dk_step *steps;
	int nsteps;
	unsigned char *blob; /* concatenated sweep programs (8-byte aligned) */
	size_t blob_bytes;
} dk_plan;

/* Planner limits (per sweep). */
typedef struct dk_plan_limits {
	int tile_bits; /* m */
	int low_bits; /* low qubits always in the tile (coalescing) */
	int max_gates;
	int max_passes;
	int max_mat; /* complex entries */
	int fuse; /* 0: one gate per sweep */
	/* Pass folding: the cost of applying one gate on its own, in FP64 FMAs
	 * per thread (8 amplitudes), against which runs of gates inside a pass
	 * are replaced by their 8x8 product.  In: 0 = default, < 0 = off.
	 * Out: the cost used, 0 = off. */
	int fold;
	/* Tensor sweeps (tiles of at least 8 qubits): in 0 = on, < 0 = off;
	 * out 1 / 0. */
	int tensor;
	/* Access pattern the bank map of a tensor sweep is chosen for: 0 the
	 * mma.sync kernels' lane layout, 1 whole columns per thread (the tcgen05
	 * complex64 kernel, 12-bit tiles). */
	int bank_mode;
} dk_plan_limits;

void dk_plan_default_limits(int prec, unsigned n, dk_plan_limits *lim);
int dk_plan_build(const dk_flat_op *ops, int nops, unsigned n, int prec,
		  const dk_plan_limits *lim, dk_plan *plan);
void dk_plan_free(dk_plan *plan);
int dk_gate_classify(const struct dk_gate *g);

/* Debug builds only (libdokigpu_dbg.so, -DDK_DEBUG_CHECKS): the first failed
 * kernel index check since the last reset, 0 if none (site in bits 56-63,
 * index in bits 0-55). */
int dk_debug_checks(uint64_t *first_failure, int reset);
/* Debug builds only: 1 starves every later tcgen05 sweep of its MMA
 * completions (its bounded waits expire: DK_ERR_TIMEOUT at the next read),
 * 0 restores normal operation. */
int dk_debug_tm_starve(int on);

#ifdef __cplusplus
}

#include <nvtx3/nvToolsExt.h>

/* An NVTX range over one C-ABI call, named after the function, so that a
 * profiler timeline (ncu --nvtx, Nsight Systems) shows which call launched
 * which kernels.  NVTX is header-only: with no tool attached a push or pop
 * is a check of one function pointer. */
struct dk_nvtx_scope {
	explicit dk_nvtx_scope(const char *name) { nvtxRangePushA(name); }
	~dk_nvtx_scope() { nvtxRangePop(); }
	dk_nvtx_scope(const dk_nvtx_scope &) = delete;
	dk_nvtx_scope &operator=(const dk_nvtx_scope &) = delete;
};
#define DK_TRACE() dk_nvtx_scope dk_nvtx_scope_(__func__)
#endif

#endif /* DK_INTERNAL_H_ */
