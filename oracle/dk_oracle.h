/*
 * CPU oracle for the Doki state-vector path -- TEST INFRASTRUCTURE ONLY.
 *
 * Restates, in plain C11 over host arrays, the arithmetic of the reference
 * engine (Mowstyl/Doki, src/doki/qops.c, qstate.{c,h}, funmatrix.c) so that
 * the CUDA path can be checked against it.  Nothing in the product links to
 * this file; only tests/, __graft_entry__.smoke() and bench.py's CPU legs do.
 *
 * Layout: a register of n qubits is 2^n complex128 amplitudes stored
 * interleaved (re, im) plus a real normalisation constant `norm`; the logical
 * amplitude i is amp[i] / norm (reference qstate.h:84-86).  Qubit q is bit q of
 * the amplitude index (LSB = qubit 0).
 *
 * Parity pinning: tests/test_oracle.py checks every function here against the
 * reference module compiled from source into oracle/_ref/, and against the
 * golden fixtures in tests/golden/ generated from that module.
 */
#ifndef DK_ORACLE_H_
#define DK_ORACLE_H_

#include <stdint.h>

/* qops.c:176-261 apply_gate: out[i] = sum_j G[row(i)][j] * (in[idx(i,j)]/in_norm)
 * when controls/anticontrols hold, else in[i]/in_norm; *out_norm = sqrt(sum |out|^2).
 * gate: 2^k x 2^k row-major complex128 (interleaved), targets[0] = LSB of row. */
int dko_apply_gate(const double *in, double in_norm, unsigned n,
		   const double *gate, unsigned k, const unsigned *targets,
		   uint64_t control_mask, uint64_t anticontrol_mask,
		   double *out, double *out_norm);

/* qops.c:72-95 probability: sum over i with bit q set of |in[i]/norm|^2. */
double dko_probability(const double *in, double norm, unsigned n, unsigned q);

/* qops.c:138-174 collapse: out[j] = in[insert(bit q = value, j)]/norm,
 * *out_norm = sqrt(value ? prob_one : 1 - prob_one).  n >= 2. */
void dko_collapse(const double *in, double norm, unsigned n, unsigned q,
		  int value, double prob_one, double *out, double *out_norm);

/* qops.c:97-122 join: out[i * 2^n2 + j] = (s1[i]/n1) * (s2[j]/n2). */
void dko_join(const double *s1, double norm1, unsigned n1, const double *s2,
	      double norm2, unsigned n2, double *out);

/* qops.c:46-70 get_global_phase: arg of the first non-zero amplitude when its
 * imaginary part is non-zero, else 0. */
double dko_global_phase(const double *in, double norm, unsigned n);

/* qops.c:266-293 + funmatrix.c:905-944: one element of the chained partial
 * trace of |psi><psi|.  elems[0..t-1] are the qubit ids passed to successive
 * funmatrix_partialtrace calls (each relative to the matrix it was applied to).
 * Evaluated by the same recursion as the reference (2^t leaves). */
void dko_ptrace_elem(const double *in, double norm, unsigned n,
		     const int *elems, unsigned t, uint64_t i, uint64_t j,
		     double *re, double *im);

/* Materialised reduced density matrix over the qubits in keep_mask:
 * rho[a][a'] = sum_b psi[a|b] conj(psi[a'|b]) / norm^2, kept qubits in
 * increasing order forming the bits of a.  out: 4^k complex128, row-major. */
void dko_reduced_density(const double *in, double norm, unsigned n,
			 uint64_t keep_mask, double *out);

/* All single-qubit marginals P(q=1), q = 0..n-1. */
void dko_marginals(const double *in, double norm, unsigned n, double *p);

#endif
