/*
 * CPU oracle for the Doki state-vector path -- TEST INFRASTRUCTURE ONLY.
 * See dk_oracle.h for the layout and the reference functions each routine
 * restates.  Written for clarity, not speed; OpenMP only shortens test time.
 */
#include "dk_oracle.h"

#include <complex.h>
#include <math.h>
#include <stddef.h>

typedef double complex cplx;

static inline cplx ld(const double *v, uint64_t i)
{
	return CMPLX(v[2 * i], v[2 * i + 1]);
}

static inline void st(double *v, uint64_t i, cplx x)
{
	v[2 * i] = creal(x);
	v[2 * i + 1] = cimag(x);
}

/* Insert bit `value` at position `bit` of `pos` (funmatrix.c:905-918 and the
 * index arithmetic of qops.c:84-93 / 164-170). */
static inline uint64_t insert_bit(uint64_t pos, unsigned bit, unsigned value)
{
	uint64_t low = pos & ((UINT64_C(1) << bit) - 1);
	return ((pos >> bit) << (bit + 1)) | ((uint64_t)value << bit) | low;
}

int dko_apply_gate(const double *in, double in_norm, unsigned n,
		   const double *gate, unsigned k, const unsigned *targets,
		   uint64_t control_mask, uint64_t anticontrol_mask,
		   double *out, double *out_norm)
{
	const uint64_t size = UINT64_C(1) << n;
	const uint64_t gsize = UINT64_C(1) << k;
	double acc = 0.0;
	int64_t i;

#pragma omp parallel for reduction(+ : acc) schedule(static)
	for (i = 0; i < (int64_t)size; i++) {
		uint64_t ui = (uint64_t)i;
		cplx sum;
		if ((ui & control_mask) == control_mask &&
		    (ui & anticontrol_mask) == 0) {
			/* row = the target bits of i, targets[0] least significant */
			uint64_t row = 0;
			for (unsigned m = 0; m < k; m++)
				row |= ((ui >> targets[m]) & 1u) << m;
			sum = 0;
			for (uint64_t col = 0; col < gsize; col++) {
				uint64_t src = ui;
				for (unsigned m = 0; m < k; m++) {
					uint64_t bit = UINT64_C(1) << targets[m];
					src = ((col >> m) & 1u) ? (src | bit)
								: (src & ~bit);
				}
				sum += (ld(in, src) / in_norm) *
				       ld(gate, row * gsize + col);
			}
		} else {
			sum = ld(in, ui) / in_norm;
		}
		st(out, ui, sum);
		acc += creal(sum) * creal(sum) + cimag(sum) * cimag(sum);
	}
	*out_norm = sqrt(acc);
	return 0;
}

double dko_probability(const double *in, double norm, unsigned n, unsigned q)
{
	const uint64_t half = UINT64_C(1) << (n - 1);
	double acc = 0.0;
	int64_t j;

#pragma omp parallel for reduction(+ : acc) schedule(static)
	for (j = 0; j < (int64_t)half; j++) {
		cplx v = ld(in, insert_bit((uint64_t)j, q, 1)) / norm;
		acc += creal(v) * creal(v) + cimag(v) * cimag(v);
	}
	return acc;
}

void dko_collapse(const double *in, double norm, unsigned n, unsigned q,
		  int value, double prob_one, double *out, double *out_norm)
{
	const uint64_t half = UINT64_C(1) << (n - 1);
	int64_t j;

#pragma omp parallel for schedule(static)
	for (j = 0; j < (int64_t)half; j++)
		st(out, (uint64_t)j,
		   ld(in, insert_bit((uint64_t)j, q, value ? 1u : 0u)) / norm);
	*out_norm = sqrt(value ? prob_one : 1.0 - prob_one);
}

void dko_join(const double *s1, double norm1, unsigned n1, const double *s2,
	      double norm2, unsigned n2, double *out)
{
	const uint64_t size1 = UINT64_C(1) << n1, size2 = UINT64_C(1) << n2;
	int64_t i;

#pragma omp parallel for schedule(static)
	for (i = 0; i < (int64_t)size1; i++) {
		cplx a = ld(s1, (uint64_t)i) / norm1;
		for (uint64_t j = 0; j < size2; j++)
			st(out, (uint64_t)i * size2 + j, a * (ld(s2, j) / norm2));
	}
}

double dko_global_phase(const double *in, double norm, unsigned n)
{
	const uint64_t size = UINT64_C(1) << n;
	for (uint64_t i = 0; i < size; i++) {
		cplx v = ld(in, i) / norm;
		if (creal(v) != 0.0 || cimag(v) != 0.0)
			return cimag(v) != 0.0 ? carg(v) : 0.0;
	}
	return 0.0;
}

static cplx ptrace_rec(const double *in, double norm, const int *elems,
		       unsigned t, uint64_t i, uint64_t j)
{
	if (t == 0)
		return (ld(in, i) / norm) * conj(ld(in, j) / norm);
	unsigned e = (unsigned)elems[t - 1];
	return ptrace_rec(in, norm, elems, t - 1, insert_bit(i, e, 0),
			  insert_bit(j, e, 0)) +
	       ptrace_rec(in, norm, elems, t - 1, insert_bit(i, e, 1),
			  insert_bit(j, e, 1));
}

void dko_ptrace_elem(const double *in, double norm, unsigned n,
		     const int *elems, unsigned t, uint64_t i, uint64_t j,
		     double *re, double *im)
{
	(void)n;
	cplx v = ptrace_rec(in, norm, elems, t, i, j);
	*re = creal(v);
	*im = cimag(v);
}

/* Scatter the bits of `val` onto the set bits of `mask` (lowest first). */
static inline uint64_t deposit(uint64_t val, uint64_t mask)
{
	uint64_t r = 0;
	for (uint64_t b = 1; mask; b <<= 1) {
		uint64_t low = mask & (~mask + 1);
		if (val & b)
			r |= low;
		mask &= mask - 1;
	}
	return r;
}

void dko_reduced_density(const double *in, double norm, unsigned n,
			 uint64_t keep_mask, double *out)
{
	const uint64_t full = (n >= 64) ? ~UINT64_C(0) : ((UINT64_C(1) << n) - 1);
	const uint64_t trace_mask = full & ~keep_mask;
	unsigned k = (unsigned)__builtin_popcountll(keep_mask);
	unsigned t = n - k;
	const uint64_t dim = UINT64_C(1) << k, tdim = UINT64_C(1) << t;
	int64_t a;

#pragma omp parallel for schedule(dynamic, 1)
	for (a = 0; a < (int64_t)dim; a++) {
		uint64_t ia = deposit((uint64_t)a, keep_mask);
		for (uint64_t a2 = 0; a2 < dim; a2++) {
			uint64_t ia2 = deposit(a2, keep_mask);
			cplx acc = 0;
			for (uint64_t b = 0; b < tdim; b++) {
				uint64_t ib = deposit(b, trace_mask);
				acc += (ld(in, ia | ib) / norm) *
				       conj(ld(in, ia2 | ib) / norm);
			}
			st(out, (uint64_t)a * dim + a2, acc);
		}
	}
}

void dko_marginals(const double *in, double norm, unsigned n, double *p)
{
	for (unsigned q = 0; q < n; q++)
		p[q] = dko_probability(in, norm, n, q);
}
