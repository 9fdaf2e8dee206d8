/*
 * dokigpu.h -- C ABI of the B200 state-vector engine behind the `doki` module.
 *
 * The entry points replace the reference engine's internal C layer (Mowstyl/Doki
 * src/doki/qstate.h, qops.h, funmatrix.h), which its CPython binding
 * (src/doki/doki.c) calls; each declaration cites the function it stands in
 * for.  Plain C types only: opaque handles, pointers, sizes, int status codes.
 * No call aborts; every failure is a non-zero status (see dk_strerror).
 *
 * Layout: a register of n qubits is 2^n amplitudes resident in device memory
 * (complex128 or complex64, interleaved re/im) plus a device-side FP64
 * normalisation constant; logical amplitude i = amp[i] / norm, exactly as the
 * reference's lazy norm (qstate.h:84-86).  Qubit q is bit q of the index.
 * Host buffers passed to or returned from this ABI are complex128 interleaved
 * (double re, double im) regardless of the register's storage precision.
 *
 * Registers are immutable values with copy-on-write storage: operations that
 * "return a new register" (apply, clone, measure) share device storage until
 * one of the sharers needs to diverge, so `r = apply(r, g)` chains run in place
 * once the previous handle is freed.  Gates queued on a register are fused
 * into multi-gate sweeps when the register is next read.
 */
#ifndef DOKIGPU_H_
#define DOKIGPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define DK_OK 0
#define DK_ERR_ALLOC 1 /* allocation failed: state_init codes 1/2, qstate.c:23-88 */
#define DK_ERR_QUBITS 3 /* too many qubits: state_init code 3, qstate.c:30-32 */
#define DK_ERR_ARG 20 /* invalid argument (range, overlap, size) */
#define DK_ERR_CUDA 21 /* a CUDA runtime call failed */
#define DK_ERR_BUDGET 22 /* the device-memory budget would be exceeded */
#define DK_ERR_TIMEOUT 23 /* a bounded device wait ran out */
#define DK_ERR_DEAD 24 /* handle was explicitly freed (registry_del) */
#define DK_ERR_EMPTY 25 /* operation on a 0-qubit register */
#define DK_ERR_NORM0 26 /* collapse produced a zero normalisation constant */
#define DK_ERR_NODEV 27 /* no usable CUDA device */
#define DK_ERR_NOALLOC_LIMIT 28 /* register larger than dk_marginals_noalloc handles */

/* ---- precisions (reference platform.h:199 PRECISION 1 / 2) ------------ */
#define DK_C64 1 /* complex64 amplitudes, FP64 norm / reductions */
#define DK_C128 2 /* complex128 amplitudes (the reference's type) */

/* Largest register the engine accepts (the reference's MAX_NUM_QUBITS is 62,
 * platform.h:270; 2^40 amplitudes already exceed any single device). */
#define DK_MAX_QUBITS 40

typedef struct dk_state dk_state;
typedef struct dk_gate dk_gate;

const char *dk_strerror(int status);
/* Text of the last CUDA error seen by this library (or ""). */
const char *dk_last_cuda_error(void);

/* Select / initialise the device for this process (default: device 0 on
 * first use).  Idempotent. */
int dk_init(int device);

/* ---- gates: struct qgate, qgate.h:25-32; gate_new doki.c:417-512 ---------
 * matrix: 2^k x 2^k row-major, complex128 interleaved.  Row index bit m is
 * the value of targets[m] (targets[0] least significant), qops.c:227-240. */
int dk_gate_new(unsigned num_qubits, const double *matrix, dk_gate **out);
/* gate_get doki.c:514-544: copy the matrix back (2 * 4^k doubles). */
int dk_gate_get(const dk_gate *gate, double *matrix);
unsigned dk_gate_num_qubits(const dk_gate *gate);
void dk_gate_free(dk_gate *gate);

/* ---- registers: struct state_vector, qstate.h:44-59 --------------------- */
/* state_init(init=1) qstate.c:23-88 via registry_new doki.c:302-341: |0..0>. */
int dk_state_new(unsigned num_qubits, int precision, dk_state **out);
/* registry_new_data doki.c:625-720: 2^n complex128 values from host memory,
 * stored as given (no normalisation; norm = 1). */
int dk_state_from_host(unsigned num_qubits, int precision,
		       const double *values, dk_state **out);
/* state_clone qstate.c:90-105 (copy-on-write: no device copy is made). */
int dk_state_clone(dk_state *src, dk_state **out);
/* registry_del doki.c:400-415: release device storage now; later use of the
 * handle returns DK_ERR_DEAD.  The handle itself stays valid until freed. */
void dk_state_release(dk_state *s);
/* state_clear qstate.c:107-121 + free: drop the handle. */
void dk_state_free(dk_state *s);
/* state_mem_size qstate.c:123-135: bytes of device + host storage. */
size_t dk_state_mem_size(const dk_state *s);
unsigned dk_state_num_qubits(const dk_state *s);
int dk_state_precision(const dk_state *s);

/* ---- the hot path: qops.h:28-56 ----------------------------------------- */
/* apply_gate qops.c:176-261: returns a new register G(controls) * in,
 * renormalised.  Targets, controls and anticontrols must be distinct and
 * < num_qubits. */
int dk_apply_gate(dk_state *in, const dk_gate *gate, const unsigned *targets,
		  unsigned num_targets, const unsigned *controls,
		  unsigned num_controls, const unsigned *anticontrols,
		  unsigned num_anticontrols, dk_state **out);

/* Bulk form of dk_apply_gate (serving form; no counterpart in the
 * reference, whose callers make one registry_apply call per gate,
 * doki.c:722-941): queue `count` gates on `in` in order and return the
 * resulting register.  Gate i acts on op_k[i] <= 3 targets
 * op_targets[3 i .. 3 i + k - 1] (targets[0] = LSB of the gate index), with
 * control / anticontrol bit masks op_controls[i] / op_anticontrols[i]; its
 * 2^k x 2^k row-major complex128 matrix starts at complex entry op_matrix[i]
 * of `matrices` (num_matrix_entries complex entries in all).  Every gate is
 * checked before any is queued; count = 0 returns a clone of `in`. */
int dk_apply_gates(dk_state *in, unsigned count, const unsigned *op_k,
		   const unsigned *op_targets, const uint64_t *op_controls,
		   const uint64_t *op_anticontrols, const uint64_t *op_matrix,
		   const double *matrices, uint64_t num_matrix_entries, dk_state **out);

/* state_get qstate.h:86 (registry_get doki.c:546-595): logical amplitude. */
int dk_get_amplitude(dk_state *s, uint64_t id, double *re, double *im);
/* Bulk form of the above: amplitudes [first, first + count) into `out`
 * (2 * count doubles). */
int dk_get_amplitudes(dk_state *s, uint64_t first, uint64_t count,
		      double *out);
/* get_global_phase qops.c:46-70: arg of the first non-zero amplitude if its
 * imaginary part is non-zero, else 0 (cached per register). */
int dk_global_phase(dk_state *s, double *phase);

/* probability qops.c:72-95: P(target = 1). */
int dk_probability(dk_state *s, unsigned target, double *p);
/* All n single-qubit marginals P(q = 1) in one sweep (p: n doubles). */
int dk_marginals(dk_state *s, double *p);

/* measure qops.c:124-136: result = P(target=1) > roll, then collapse
 * (qops.c:138-174) into a register one qubit smaller (*out = NULL when the
 * input had one qubit). */
int dk_measure(dk_state *s, unsigned target, double roll, int *result,
	       dk_state **out);
/* registry_measure doki.c:1023-1192: qubits num_qubits-1 .. 0 that are set in
 * `mask`, one roll each in that order (rolls must be in [0, 1)).  results:
 * num_qubits entries, results[i] for qubit num_qubits-1-i: -1 = not
 * measured, 0 / 1 = outcome.  *out = NULL when every qubit was measured. */
int dk_measure_mask(dk_state *s, uint64_t mask, const double *rolls,
		    unsigned num_rolls, int8_t *results, dk_state **out);

/* ---- distributed registers (no counterpart in the reference) ------------
 * The local part of a register sharded over ranks by its top qubits: each
 * rank holds a register of the low qubits, and a gate on a rank qubit swaps
 * that qubit with a local one by exchanging half of the local amplitudes
 * with the partner rank.  These three calls give the rank its local view. */
/* Once the queued gates of `s` have run: its norm constant (logical
 * amplitude = stored amplitude / norm) and the 2-norm of its stored
 * amplitudes (equal after a gate; a register stored as given keeps norm 1). */
int dk_state_norm(dk_state *s, double *norm, double *stored_norm);
/* scale x the logical amplitudes of `s` whose qubit `bit` equals `value`
 * (2^(n-1) of them, in index order) into `dst`, in the register's storage
 * precision (complex64 or complex128, interleaved); `dst` is device memory
 * when on_device, else host memory (then the call waits for the copy). */
int dk_state_read_half(dk_state *s, unsigned bit, int value, double scale, void *dst,
		       int on_device);
/* A new register: its amplitudes with qubit `bit` = `value` are `src`
 * (2^(n-1), storage precision, index order; device memory when on_device),
 * the others are scale x the logical amplitudes of `in`; stored as given
 * (norm 1), like dk_state_from_host. */
int dk_state_replace_half(dk_state *in, unsigned bit, int value, double scale, const void *src,
			  int on_device, dk_state **out);

/* join qops.c:97-122: tensor product, `most` on the high qubits. */
int dk_join(dk_state *most, dk_state *least, dk_state **out);

/* density_matrix qops.c:580-601 followed by partial_trace funmatrix.c:999-1037
 * over every qubit outside keep_mask, materialised: out[a * 2^k + a'] =
 * sum_b psi[a|b] conj(psi[a'|b]) with the k kept qubits, in increasing order,
 * forming the bits of a.  out: 2 * 4^k doubles, k <= 14. */
int dk_reduced_density(dk_state *s, uint64_t keep_mask, double *out);
/* One element of the same matrix, for kept sets too large to materialise. */
int dk_reduced_density_elem(dk_state *s, uint64_t keep_mask, uint64_t i,
			    uint64_t j, double *re, double *im);

/* Precision form (no counterpart in the reference): fidelity
 * |<x|y>|^2 of the two logical (normalised) registers and the largest
 * |x_i - y_i|, accumulated in FP64; x and y may have different precisions. */
int dk_compare_states(dk_state *x, dk_state *y, double *fidelity, double *max_amp_err);

/* Wait for all queued device work of this library. */
int dk_sync(void);

/* ---- engine controls (no counterpart in the reference) ------------------ */
/* 1 (default): queued gates are fused into multi-gate sweeps when a register
 * is read; 0: every gate is its own sweep (the per-gate plain method). */
int dk_set_fusion(int enable);
/* Counters since dk_init: CUDA kernels launched by this library, fused
 * sweeps executed and gates applied by them.  Any pointer may be NULL. */
int dk_get_stats(uint64_t *kernel_launches, uint64_t *sweeps,
		 uint64_t *gates_applied);
/* Tensor-core sweep work since dk_init: the sum over launched tensor sweeps
 * of (8x8 matrix entries in the sweep) x (amplitudes of the register).  One
 * entry-amplitude is 24 FMA on FP64 MMAs (complex128, Gauss form: 3 real
 * products of 2 m8n8k4 k-steps per 64 amplitudes) or 96 TF32 MMA FMA
 * (complex64: 6 m16n8k8 MMAs per 64 amplitudes). */
int dk_get_mma_stats(uint64_t *entry_amplitudes);
/* complex64 sweeps launched on tcgen05 since load: with every B operand of
 * the sweep split once per CTA into shared memory, and with B split per
 * entry (sweeps whose matrices do not fit, or DK_C64_TMEM_PRESPLIT=0). */
int dk_get_tm_stats(uint64_t *presplit, uint64_t *per_entry);
/* Bytes copied host->device and device->host by this library since dk_init. */
int dk_get_io_stats(uint64_t *h2d_bytes, uint64_t *d2h_bytes);
/* Execute the gates queued on `s` now (normally deferred to the next read). */
int dk_state_flush(dk_state *s);
/* The CUDA stream (cudaStream_t) of the calling thread's slot, for callers
 * that time its work with events; NULL before initialisation. */
void *dk_stream(void);

/* ---- slots: concurrent streams (no counterpart in the reference) --------
 * A slot is a CUDA stream with its own scratch.  Registers are created on the
 * calling thread's current slot (0 unless dk_slot_set was called) and every
 * register derived from one stays on its slot; work of different slots runs
 * concurrently on the device and each slot has its own lock, so threads that
 * drive different slots do not wait for each other.  Up to 64 slots. */
int dk_slot_new(int *slot);
int dk_slot_set(int slot);
int dk_slot_get(void);

/* ---- batching form (no counterpart in the reference) --------------------
 * Thousands of independent registers (4..16 qubits), each starting in |0..0>
 * with its own gate sequence, run by one CUDA-graph launch.  Circuit c has
 * num_qubits[c] qubits and ops op_start[c] .. op_start[c+1]-1; op i acts on
 * op_k[i] <= 3 targets op_targets[3*i .. 3*i+k-1] (targets[0] = LSB of the
 * gate index, as registry_apply), with control / anticontrol bit masks
 * op_controls[i] / op_anticontrols[i], and its 2^k x 2^k row-major complex128
 * matrix starts at complex entry op_matrix[i] of `matrices`.  Dense 3-qubit
 * gates are not accepted (diagonal ones are).  After the circuit, each
 * register's reduced density matrix over its lower keep_qubits[c] qubits
 * (<= 12) is formed on the device, divided by its trace.  Registers above 12
 * qubits stream through tiles of `tile_bits` (8..12) qubits. */
typedef struct dk_batch dk_batch;
int dk_batch_build(int precision, unsigned num_circuits, const unsigned *num_qubits,
		   const unsigned *keep_qubits, const uint64_t *op_start,
		   const unsigned *op_k, const unsigned *op_targets,
		   const uint64_t *op_controls, const uint64_t *op_anticontrols,
		   const uint64_t *op_matrix, const double *matrices, int tile_bits,
		   int fold, dk_batch **out);
/* `fold` is the dense-block fusion of the plan: a run of gates inside a
 * 3-qubit pass becomes one 8x8 product when that costs less than applying
 * them one by one, each gate charged its arithmetic plus `fold` FP64
 * multiply-adds per thread of dispatch; 0 = the planner's default (96),
 * < 0 = off (every gate applied on its own), larger values fold more
 * readily.  The circuits are planned on all host cores.
 * CTAs per SM for the batch kernels (1..4); the autotuner's second knob. */
int dk_batch_set_ctas(dk_batch *b, int ctas_per_sm);
/* Queue every circuit (captured into a CUDA graph on first use); keep_states
 * also stores each final register for dk_batch_state.  Returns before the
 * device finishes; see dk_batch_sync / dk_batch_stream. */
int dk_batch_run(dk_batch *b, int keep_states);
int dk_batch_sync(dk_batch *b);
void *dk_batch_stream(dk_batch *b);
/* reduced density matrix of circuit c: 2 * 4^keep doubles (row-major) */
int dk_batch_rho(dk_batch *b, unsigned circuit, double *out);
/* all reduced density matrices, concatenated; offsets[c] = first complex
 * entry of circuit c (may be NULL) */
int dk_batch_rho_all(dk_batch *b, double *out, uint64_t *offsets);
uint64_t dk_batch_rho_elems(const dk_batch *b);
/* final raw amplitudes of circuit c (needs keep_states): 2 * 2^n doubles */
int dk_batch_state(dk_batch *b, unsigned circuit, double *out);
/* Precision form of the batch: for every circuit of two batches built from
 * the same circuits (typically complex64 and complex128), both run with
 * keep_states, the fidelity |<x|y>|^2 / (<x|x> <y|y>) of the final registers
 * and the largest |x_i / |x| - y_i / |y||, computed on the device in FP64
 * (fidelity, max_amp_err: one double per circuit). */
int dk_batch_compare(dk_batch *x, dk_batch *y, double *fidelity, double *max_amp_err);
const char *dk_batch_error(const dk_batch *b);
/* Host seconds dk_batch_build spent planning the circuits (on all host
 * threads), assembling the program blob and register tables, and allocating
 * and uploading the device buffers. */
int dk_batch_build_times(const dk_batch *b, double *plan_s, double *assemble_s,
			 double *upload_s);
void dk_batch_free(dk_batch *b);

/* ---- allocation-free marginals (no counterpart in the reference) --------
 * For callers that cannot let a library allocate device memory (a framework
 * that owns every device byte through its own allocator or an HBM-budget
 * arena, or a latency-critical loop where cudaMalloc / cudaFree would
 * synchronise the device).  Same reduction as dk_marginals, on a caller-owned
 * device array `amps` of 2^num_qubits amplitudes (complex64 or complex128 by
 * `precision`), queued on `stream` (a cudaStream_t, NULL = default stream).
 * Writes num_qubits + 1 doubles to the caller-owned device array `out`:
 * out[q] = sum of |amps[i]|^2 over i with bit q set, out[num_qubits] = the
 * sum over all i.  Allocates nothing: its scratch is a fixed 128 KiB array in
 * every device that loads this library, held until the process exits.  The
 * first call on a device looks that array's device address up (make it before
 * any stream capture).  Calls share the array, so calls that overlap on the
 * device race.  num_qubits above DK_NOALLOC_MAX_QUBITS returns
 * DK_ERR_NOALLOC_LIMIT. */
#define DK_NOALLOC_MAX_QUBITS 40
int dk_marginals_noalloc(const void *amps, unsigned num_qubits, int precision,
			 double *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* DOKIGPU_H_ */
