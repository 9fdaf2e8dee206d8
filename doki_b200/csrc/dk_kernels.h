/* Launch wrappers of the engine's CUDA kernels (internal, C++). */
#ifndef DK_KERNELS_H_
#define DK_KERNELS_H_

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

#include "dk_internal.h"

namespace dk {

/* Kernels launched by the wrappers below (for the engine's counters).
 * Several slot threads launch at once, so the count is atomic: it orders
 * nothing, it only must not lose increments. */
extern std::atomic<unsigned long long> g_launches;
/* complex64 tensor sweeps of 12-bit tiles on tcgen05 (1, default) or on the
 * mma.sync split-TF32 kernel (0) */
extern int g_c64_tmem;
/* set once a tcgen05 sweep has been launched (tm_fault_check has work) */
extern std::atomic<int> g_tm_ran;
/* tcgen05 sweeps may split all of a sweep's B operands once per CTA (1,
 * default) or must split them per entry (0) */
extern int g_tm_allow_presplit;
/* tcgen05 sweeps launched with B split once per CTA / per entry */
extern std::atomic<unsigned long long> g_tm_presplit, g_tm_entry_b;

/* Faults counted by tcgen05 sweeps whose bounded waits expired since the
 * last call (0 = none); reads and clears the device counter on `st`. */
cudaError_t tm_fault_check(cudaStream_t st, unsigned *faults);

/* Number of per-block partial slots the scratch buffer must hold. */
constexpr int kMaxBlocks = 4096;
/* doubles per partial slot (marginals need n + 1 <= 64) */
constexpr int kPartialStride = 64;

struct Scratch {
	double *partials; /* kMaxBlocks * kPartialStride doubles */
	unsigned long long *u64; /* 4 words */
	double *marg; /* 64 doubles: marginal sums + total */
};

/* fused sweep: in may equal out (in place) */
cudaError_t launch_sweep(int prec, const void *in, void *out,
			 const unsigned char *dprog, const dk_sweep_hdr *hprog,
			 const dk_scal *sc_in, dk_scal *sc_out,
			 const Scratch &s, int num_sms, cudaStream_t st);

/* generic k-qubit gate, out of place */
cudaError_t launch_generic_gate(int prec, const void *in, void *out,
				unsigned n, unsigned k, const unsigned *tg,
				uint64_t cm, uint64_t am, const double *dmat,
				const dk_scal *sc_in, dk_scal *sc_out,
				const Scratch &s, cudaStream_t st);

/* distributed registers: scale x the half of `in` (raw amplitudes) at
 * bit = value into dst (2^(n-1), storage precision) */
cudaError_t launch_read_half(int prec, const void *in, unsigned n, unsigned bit, int value,
			     double scale, void *dst, cudaStream_t st);
/* out = in with its half at bit = value taken from src and the rest scaled
 * by `scale`; out's scalars: csq = sum |out|^2, norm = 1 */
cudaError_t launch_replace_half(int prec, const void *in, const void *src, unsigned n,
				unsigned bit, int value, double scale, void *out, dk_scal *sc,
				const Scratch &s, cudaStream_t st);

/* |0..0>: zero + amp[0] = 1, norm = csq = 1 */
cudaError_t launch_init_zero(int prec, void *d, unsigned n, dk_scal *sc,
			     cudaStream_t st);

/* convert host-staged complex128 into the buffer's precision (d may alias
 * src for complex128) and set norm = 1, csq = sum |x|^2 */
cudaError_t launch_import(int prec, const double *src, void *d, unsigned n,
			  dk_scal *sc, const Scratch &s, cudaStream_t st);

/* all marginal sums S_q (q < n) and the total into s.marg[0..n] */
cudaError_t launch_marginals(int prec, const void *d, unsigned n,
			     const Scratch &s, cudaStream_t st);

/* the same reduction with at most `max_blocks` (a power of two) blocks, for
 * callers whose partials array holds only that many slots */
cudaError_t launch_marginals_blocks(int prec, const void *d, unsigned n,
				    const Scratch &s, int max_blocks, cudaStream_t st);

/* decide outcome of qubit q against roll (uses s.marg), then gather the
 * selected half into out (n-1 qubits) */
cudaError_t launch_measure_collapse(int prec, const void *in, void *out,
				    unsigned n, unsigned q, double roll,
				    int forced, const dk_scal *sc_in,
				    dk_scal *sc_out, const Scratch &s,
				    cudaStream_t st);

/* Measurement of the k = popcount(mask) <= kJointMaxQubits qubits of mask,
 * highest first, in one pass: joint distribution, sequential outcomes with
 * the device rolls rolls_dev[0..k) (flags_dev[s] = outcome of step s),
 * then, when out is not null, one gather of the 2^(n-k) selected
 * amplitudes with norm = norm_in * sqrt(P(outcomes)). */
constexpr int kJointMaxQubits = 12;
constexpr uint64_t kJointPartials = 131072; /* doubles of s.partials used */
cudaError_t launch_measure_joint(int prec, const void *in, void *out, unsigned n,
				 uint64_t mask, const double *rolls_dev, int32_t *flags_dev,
				 const dk_scal *sc_in, dk_scal *sc_out, const Scratch &s,
				 cudaStream_t st);

/* out = (most / n1) (x) (least / n2), norm 1 */
cudaError_t launch_join(int prec, const void *most, unsigned n1,
			const dk_scal *sc1, const void *least, unsigned n2,
			const dk_scal *sc2, void *out, dk_scal *sc_out,
			const Scratch &s, cudaStream_t st);

/* smallest index in [first, first+count) with a non-zero amplitude, or
 * UINT64_MAX, into s.u64[0] */
cudaError_t launch_first_nonzero(int prec, const void *d, uint64_t first,
				 uint64_t count, const Scratch &s,
				 cudaStream_t st);

/* gather psi into a complex128 matrix M[b][a] (a = kept bits, b = traced) */
cudaError_t launch_gather_kept(int prec, const void *d, unsigned n,
			       uint64_t keep_mask, double2 *M, cudaStream_t st);

/* rho = alpha X X^H (X[a][b] = A[b * dim + a]) into the lower triangle of
 * the column-major C; nsplit = rho_splits(...) partials of dim * dim each
 * in part (unused when nsplit == 1 and dim >= 64) */
int rho_splits(uint64_t dim, uint64_t K, int num_sms);
cudaError_t launch_rho(const double2 *A, uint64_t dim, uint64_t K, double alpha, int nsplit,
		       double2 *part, double2 *C, cudaStream_t st);

/* lower triangle of the column-major Hermitian C -> full row-major rho */
cudaError_t launch_herm_fill(const double2 *C, double2 *rho, uint64_t dim,
			     cudaStream_t st);

/* one reduced-density element, summed into s.marg[0..1] */
cudaError_t launch_rho_elem(int prec, const void *d, unsigned n,
			    uint64_t keep_mask, uint64_t i, uint64_t j,
			    const dk_scal *sc, const Scratch &s,
			    cudaStream_t st);

/* copy amplitudes [first, first+count) to complex128 dst (device) */
cudaError_t launch_export(int prec, const void *d, uint64_t first,
			  uint64_t count, double2 *dst, cudaStream_t st);

/* fidelity terms of two registers: s.marg[0..2] = Re, Im of sum conj(sx x)
 * (sy y) and max |sx x - sy y| */
cudaError_t launch_compare(int prec_x, const void *x, double sx, int prec_y, const void *y,
			   double sy, unsigned n, const Scratch &s, cudaStream_t st);

/* D2D copy of a register (clone that must diverge), scalars included */
cudaError_t launch_copy(int prec, const void *src, void *dst, unsigned n,
			const dk_scal *sc_in, dk_scal *sc_out,
			cudaStream_t st);

} // namespace dk

#endif
