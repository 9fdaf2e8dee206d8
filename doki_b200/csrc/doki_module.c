/*
 * doki -- CPython extension with the reference module's API (Mowstyl/Doki
 * src/doki/doki.c), backed by the B200 engine's C ABI (include/dokigpu.h).
 *
 * Same function names, positional argument formats, capsule names
 * ("qsimov.doki.state_vector", "qsimov.doki.gate", "qsimov.doki.funmatrix"),
 * exception object (qsimov.doki.error) and error strings as the reference
 * binding.  Differences, all strictly safer: out-of-range ids (registry_get,
 * registry_prob, funmatrix_partialtrace) and repeated targets raise instead
 * of reading out of bounds; a registry passed to registry_del raises on
 * later use instead of being a dangling pointer; custom matrices of any shape
 * are stored row-major (the reference indexes them with the row count);
 * funmatrix_projection and funmatrix_apply honour their qubit id and state
 * arguments (the reference's wrappers store "p" ints into 1-byte bools next
 * to them).
 *
 * Extensions (optional trailing arguments never break positional calls):
 *   registry_new(n, verbose[, precision]) / registry_new_data(n, values,
 *   verbose[, precision]) -- precision 2 = complex128 (default), 1 = complex64;
 *   registry_get_all(reg, canonical) -> numpy complex128 array;
 *   registry_probs(reg) -> list of all P(q = 1);
 *   funmatrix_numpy(fm) -> numpy array of any functional matrix (one device
 *   call for a reduced density matrix);
 *   registry_precision(reg); registry_flush(reg); registry_compare(a, b);
 *   engine_sync();
 *   engine_set_fusion(bool); engine_stats(); engine_stream();
 *   engine_new_slot(); engine_set_slot(slot); engine_get_slot();
 *   registry_apply_many(reg, op_k, op_targets, op_controls, op_anticontrols,
 *   op_matrix, matrices) -- a whole circuit in one call (serving form);
 *   registry_norm(reg), registry_read_half(...), registry_replace_half(...)
 *   -- the local view of a distributed register (doki_b200.dist).
 */
#define PY_SSIZE_T_CLEAN
#include <Python.h>
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "dokigpu.h"

static PyObject *DokiError;
static PyObject *np_mod, *np_ndarray, *np_complex128;

#define CAP_STATE "qsimov.doki.state_vector"
#define CAP_GATE "qsimov.doki.gate"
#define CAP_FMAT "qsimov.doki.funmatrix"

#define THREADS_MSG "num_threads must be at least 1 (or -1 to let OpenMP choose)"

static PyObject *raise_dk(int rc, const char *ctx)
{
	const char *cu = dk_last_cuda_error();
	if (rc == DK_ERR_CUDA && cu && cu[0])
		PyErr_Format(DokiError, "%s: %s (%s)", ctx, dk_strerror(rc), cu);
	else
		PyErr_Format(DokiError, "%s: %s", ctx, dk_strerror(rc));
	return NULL;
}

static dk_state *get_state(PyObject *cap, const char *msg)
{
	dk_state *s = (dk_state *)PyCapsule_GetPointer(cap, CAP_STATE);
	if (s == NULL)
		PyErr_SetString(DokiError, msg);
	return s;
}

static void state_destroy(PyObject *cap)
{
	dk_state *s = (dk_state *)PyCapsule_GetPointer(cap, CAP_STATE);
	if (s)
		dk_state_free(s);
	else
		PyErr_Clear();
}

static void gate_destroy(PyObject *cap)
{
	dk_gate *g = (dk_gate *)PyCapsule_GetPointer(cap, CAP_GATE);
	if (g)
		dk_gate_free(g);
	else
		PyErr_Clear();
}

static PyObject *wrap_state(dk_state *s)
{
	PyObject *c = PyCapsule_New(s, CAP_STATE, state_destroy);
	if (!c)
		dk_state_free(s);
	return c;
}

/* ======================= functional matrices ============================ */

/* Node kinds.  Every node carries the reference's per-node modifiers
 * (funmatrix.h struct FMatrix): a scalar s, a transpose flag and a conjugate
 * flag, applied by fmat_get around the kind's own element rule. */
enum {
	FM_CUSTOM = 1,
	FM_IDENTITY,
	FM_STATEZERO,
	FM_DENSITYZERO,
	FM_WALSH,
	FM_CU,
	FM_DENSITY,
	FM_PTRACE,
	FM_EYEKRON,
	FM_PROJECTION,
	FM_APPLY,
	/* operation nodes A op B (funmatrix.h op codes 0-4) */
	FM_ADD,
	FM_SUB,
	FM_MATMUL,
	FM_EWMUL,
	FM_KRON,
};

/* Element status codes of the reference's getitem (funmatrix.c:238-340),
 * offset by 100 so they never collide with DK_* codes. */
enum {
	FMG_ADD = 101,
	FMG_SUB,
	FMG_MATMUL,
	FMG_EWMUL,
	FMG_KRON,
	FMG_OP,
	FMG_BOUNDS,
	FMG_NAN,
};

/* Host array of a custom matrix, shared by the copies that scalar products,
 * transposes and daggers make. */
typedef struct fm_buf {
	size_t refs;
	size_t len;
	double complex v[];
} fm_buf;

typedef struct fmat {
	int kind;
	uint64_t r, c;
	double complex s;
	int transpose, conjugate;
	/* A and B of operation nodes; the operand of CU, PTRACE, EYEKRON and
	 * PROJECTION (a); state and gate of APPLY; the state capsule of DENSITY */
	PyObject *a, *b;
	int elem; /* PTRACE: traced qubit; PROJECTION: qubit id */
	int value; /* PROJECTION: kept value of the qubit */
	uint64_t left, right; /* EYEKRON: identity sizes 2^leftQ, 2^rightQ */
	int hadamard;
	fm_buf *data; /* CUSTOM, row-major r x c */
	unsigned *targets; /* APPLY */
	unsigned ntargets;
	uint64_t cmask, amask;
	/* PTRACE chains rooted at a register: materialised reduced density */
	int mat_ready;
	uint64_t keep_mask;
	double complex *rho;
} fmat;

static void fm_buf_release(fm_buf *b)
{
	if (b && --b->refs == 0)
		free(b);
}

static void fmat_free(fmat *m)
{
	Py_XDECREF(m->a);
	Py_XDECREF(m->b);
	fm_buf_release(m->data);
	free(m->targets);
	free(m->rho);
	free(m);
}

static void fmat_destroy(PyObject *cap)
{
	fmat *m = (fmat *)PyCapsule_GetPointer(cap, CAP_FMAT);
	if (!m) {
		PyErr_Clear();
		return;
	}
	fmat_free(m);
}

static PyObject *wrap_fmat(fmat *m)
{
	PyObject *c = PyCapsule_New(m, CAP_FMAT, fmat_destroy);
	if (!c)
		fmat_free(m);
	return c;
}

static fmat *fmat_new(int kind, uint64_t r, uint64_t c)
{
	fmat *m = (fmat *)calloc(1, sizeof(fmat));
	if (m) {
		m->kind = kind;
		m->r = r;
		m->c = c;
		m->s = 1.0;
	}
	return m;
}

/* A node that evaluates like m with its own modifiers (mprod, mdiv,
 * transpose and dagger, funmatrix.c:428-860): operands and custom data are
 * shared, the reduced-density cache is not. */
static fmat *fmat_copy(const fmat *m)
{
	fmat *d = fmat_new(m->kind, m->r, m->c);
	if (!d)
		return NULL;
	if (m->targets) {
		d->targets = (unsigned *)malloc(sizeof(unsigned) * (m->ntargets ? m->ntargets : 1));
		if (!d->targets) {
			free(d);
			return NULL;
		}
		memcpy(d->targets, m->targets, sizeof(unsigned) * m->ntargets);
	}
	d->s = m->s;
	d->transpose = m->transpose;
	d->conjugate = m->conjugate;
	d->a = m->a;
	Py_XINCREF(d->a);
	d->b = m->b;
	Py_XINCREF(d->b);
	d->elem = m->elem;
	d->value = m->value;
	d->left = m->left;
	d->right = m->right;
	d->hadamard = m->hadamard;
	d->data = m->data;
	if (d->data)
		d->data->refs++;
	d->ntargets = m->ntargets;
	d->cmask = m->cmask;
	d->amask = m->amask;
	return d;
}

static fmat *fmat_of(PyObject *cap)
{
	fmat *m = cap ? (fmat *)PyCapsule_GetPointer(cap, CAP_FMAT) : NULL;
	if (!m)
		PyErr_Clear();
	return m;
}

static int fmat_plain(const fmat *m)
{
	return m->s == 1.0 && !m->transpose && !m->conjugate;
}

static uint64_t ins_bit(uint64_t pos, int e, int v)
{
	/* funmatrix.c:905-918: insert bit v at position e */
	const uint64_t aux = 1ull << e;
	return pos % aux + (pos / aux) * (aux << 1) + (uint64_t)v * aux;
}

static int ilog2(uint64_t x)
{
	int l = 0;
	while (l < 64 && (1ull << l) < x)
		l++;
	return l;
}

/* If the chain of partial traces below m ends at a register's density
 * matrix and no node on the way carries a modifier, return the state
 * capsule and the surviving-qubit mask. */
static PyObject *ptrace_root(fmat *m, uint64_t *keep)
{
	int elems[64], ne = 0;
	fmat *cur = m;
	while (cur->kind == FM_PTRACE && ne < 64) {
		elems[ne++] = cur->elem;
		cur = fmat_of(cur->a);
		if (!cur || !fmat_plain(cur))
			return NULL;
	}
	if (cur->kind != FM_DENSITY)
		return NULL;
	dk_state *s = (dk_state *)PyCapsule_GetPointer(cur->a, CAP_STATE);
	if (!s) {
		PyErr_Clear();
		return NULL;
	}
	unsigned n = dk_state_num_qubits(s);
	int alive[64];
	int na = (int)n;
	for (int q = 0; q < na; q++)
		alive[q] = q;
	/* elems were collected outermost first; apply innermost first */
	for (int t = ne - 1; t >= 0; t--) {
		int e = elems[t];
		if (e < 0 || e >= na)
			return NULL;
		memmove(alive + e, alive + e + 1, sizeof(int) * (size_t)(na - e - 1));
		na--;
	}
	uint64_t k = 0;
	for (int i = 0; i < na; i++)
		k |= 1ull << alive[i];
	*keep = k;
	return cur->a;
}

static int fmat_get(fmat *m, uint64_t i, uint64_t j, double complex *out);

/* A child element inside a functional node: a failing child makes the node's
 * value NaN in the reference (its getitem leaves NaN behind), which the
 * caller reports as FMG_NAN; engine errors pass through. */
static int child_get(PyObject *cap, uint64_t i, uint64_t j, double complex *out)
{
	fmat *c = fmat_of(cap);
	if (!c)
		return FMG_NAN;
	int rc = fmat_get(c, i, j, out);
	return rc >= FMG_ADD ? FMG_NAN : rc;
}

/* Two operand elements of an operation node; any operand failure becomes
 * the node's own code. */
static int op_get(fmat *m, uint64_t ia, uint64_t ja, uint64_t ib, uint64_t jb,
		  double complex *x, double complex *y, int code)
{
	fmat *A = fmat_of(m->a), *B = fmat_of(m->b);
	if (!A || !B)
		return code;
	int r1 = fmat_get(A, ia, ja, x);
	int r2 = fmat_get(B, ib, jb, y);
	if (r1 && r1 < FMG_ADD)
		return r1;
	if (r2 && r2 < FMG_ADD)
		return r2;
	return (r1 || r2) ? code : 0;
}

/* The kind's element rule at (i, j), after the node's transpose swap. */
static int fmat_elem(fmat *m, uint64_t i, uint64_t j, double complex *out)
{
	double complex x, y;
	int rc;
	switch (m->kind) {
	case FM_CUSTOM:
		*out = m->data->v[i * m->c + j];
		return 0;
	case FM_IDENTITY:
		*out = (i == j) ? 1.0 : 0.0;
		return 0;
	case FM_STATEZERO:
		*out = (i == 0) ? 1.0 : 0.0;
		return 0;
	case FM_DENSITYZERO:
		*out = (i == 0 && j == 0) ? 1.0 : 0.0;
		return 0;
	case FM_WALSH: {
		/* funmatrix.c:1135-1192: (-1)^popcount(i & j), / sqrt(size) for H */
		double v = (__builtin_popcountll(i & j) & 1) ? -1.0 : 1.0;
		if (m->hadamard)
			v /= sqrt((double)m->r);
		*out = v;
		return 0;
	}
	case FM_CU: {
		/* funmatrix.c:1194-1219: identity block, then U in the last block */
		fmat *u = fmat_of(m->a);
		if (!u)
			return FMG_NAN;
		if (i < u->r || j < u->c) {
			*out = (i == j) ? 1.0 : 0.0;
			return 0;
		}
		return child_get(m->a, i - u->r, j - u->c, out);
	}
	case FM_DENSITY: {
		/* qops.c:266-293: psi_i conj(psi_j) */
		dk_state *s = (dk_state *)PyCapsule_GetPointer(m->a, CAP_STATE);
		if (!s) {
			PyErr_Clear();
			return DK_ERR_ARG;
		}
		double ar, ai, br, bi;
		rc = dk_get_amplitude(s, i, &ar, &ai);
		if (!rc)
			rc = dk_get_amplitude(s, j, &br, &bi);
		if (rc)
			return rc;
		*out = (ar + I * ai) * conj(br + I * bi);
		return 0;
	}
	case FM_PTRACE: {
		if (m->mat_ready) {
			*out = m->rho[i * m->r + j];
			return 0;
		}
		uint64_t keep = 0;
		PyObject *root = ptrace_root(m, &keep);
		if (root) {
			dk_state *s = (dk_state *)PyCapsule_GetPointer(root, CAP_STATE);
			const int k = __builtin_popcountll(keep);
			if (k <= 12) {
				uint64_t dim = 1ull << k;
				double complex *rho =
					(double complex *)malloc(sizeof(double complex) * dim * dim);
				if (!rho)
					return DK_ERR_ALLOC;
				rc = dk_reduced_density(s, keep, (double *)rho);
				if (rc) {
					free(rho);
					return rc;
				}
				m->rho = rho;
				m->keep_mask = keep;
				m->mat_ready = 1;
				*out = rho[i * dim + j];
				return 0;
			}
			double re, im;
			rc = dk_reduced_density_elem(s, keep, i, j, &re, &im);
			if (rc)
				return rc;
			*out = re + I * im;
			return 0;
		}
		/* generic lazy partial trace (funmatrix.c:920-944) */
		rc = child_get(m->a, ins_bit(i, m->elem, 0), ins_bit(j, m->elem, 0), &x);
		if (!rc)
			rc = child_get(m->a, ins_bit(i, m->elem, 1), ins_bit(j, m->elem, 1), &y);
		if (rc)
			return rc;
		*out = x + y;
		return 0;
	}
	case FM_EYEKRON: {
		/* funmatrix.c:665-707: I(2^left) (x) U (x) I(2^right) */
		fmat *u = fmat_of(m->a);
		if (!u)
			return FMG_NAN;
		if (i % m->right != j % m->right) {
			*out = 0.0;
			return 0;
		}
		i /= m->right;
		j /= m->right;
		if (i / u->r != j / u->c) {
			*out = 0.0;
			return 0;
		}
		return child_get(m->a, i % u->r, j % u->c, out);
	}
	case FM_PROJECTION: {
		/* funmatrix.c:862-890: rows whose qubit differs from value are 0 */
		const int bit = (i >> m->elem) & 1;
		if (bit != m->value) {
			*out = 0.0;
			return 0;
		}
		return child_get(m->a, i, j, out);
	}
	case FM_APPLY: {
		/* qops.c:498-563: controlled gate applied to a column vector */
		if ((i & m->cmask) != m->cmask || (i & m->amask))
			return child_get(m->a, i, 0, out);
		fmat *g = fmat_of(m->b);
		if (!g)
			return FMG_NAN;
		uint64_t row = 0, reg = i;
		for (unsigned k = 0; k < m->ntargets; k++)
			row |= ((i >> m->targets[k]) & 1ull) << k;
		double complex acc = 0.0;
		for (uint64_t n = 0; n < g->r; n++) {
			for (unsigned k = 0; k < m->ntargets; k++) {
				const uint64_t tb = 1ull << m->targets[k];
				reg = ((n >> k) & 1ull) ? (reg | tb) : (reg & ~tb);
			}
			rc = child_get(m->a, reg, 0, &x);
			if (!rc)
				rc = child_get(m->b, row, n, &y);
			if (rc)
				return rc;
			acc = acc + x * y;
		}
		*out = acc;
		return 0;
	}
	case FM_ADD:
		rc = op_get(m, i, j, i, j, &x, &y, FMG_ADD);
		if (!rc)
			*out = x + y;
		return rc;
	case FM_SUB:
		rc = op_get(m, i, j, i, j, &x, &y, FMG_SUB);
		if (!rc)
			*out = x - y;
		return rc;
	case FM_MATMUL: {
		fmat *A = fmat_of(m->a);
		if (!A)
			return FMG_MATMUL;
		double complex acc = 0.0;
		for (uint64_t k = 0; k < A->c; k++) {
			rc = op_get(m, i, k, k, j, &x, &y, FMG_MATMUL);
			if (rc)
				return rc;
			acc = acc + x * y;
		}
		*out = acc;
		return 0;
	}
	case FM_EWMUL:
		rc = op_get(m, i, j, i, j, &x, &y, FMG_EWMUL);
		if (!rc)
			*out = x * y;
		return rc;
	case FM_KRON: {
		fmat *B = fmat_of(m->b);
		if (!B)
			return FMG_KRON;
		rc = op_get(m, i / B->r, j / B->c, i % B->r, j % B->c, &x, &y, FMG_KRON);
		if (!rc)
			*out = x * y;
		return rc;
	}
	default:
		return FMG_OP;
	}
}

/* Element (i, j) as the reference's getitem computes it: bounds, transpose
 * swap, the kind's rule (NaN from a functional node is an error), conjugate,
 * then the node's scalar.  Returns 0, an FMG_* code or a DK status (Python
 * error not set). */
static int fmat_get(fmat *m, uint64_t i, uint64_t j, double complex *out)
{
	*out = NAN;
	if (i >= m->r || j >= m->c)
		return FMG_BOUNDS;
	if (m->transpose) {
		const uint64_t t = i;
		i = j;
		j = t;
	}
	double complex v = NAN;
	int rc = fmat_elem(m, i, j, &v);
	if (rc)
		return rc;
	if (m->kind < FM_ADD && (isnan(creal(v)) || isnan(cimag(v)))) {
		*out = v;
		return FMG_NAN;
	}
	if (m->conjugate)
		v = conj(v);
	*out = v * m->s;
	return 0;
}

/* ============================ gates ===================================== */

static int py_to_complex(PyObject *v, double complex *out)
{
	/* doki.c:484-496: complex, float or int */
	if (PyComplex_Check(v))
		*out = PyComplex_RealAsDouble(v) + I * PyComplex_ImagAsDouble(v);
	else if (PyFloat_Check(v))
		*out = PyFloat_AsDouble(v);
	else if (PyLong_Check(v))
		*out = (double)PyLong_AsLong(v);
	else
		return -1;
	return 0;
}

static PyObject *doki_gate_new(PyObject *self, PyObject *args)
{
	PyObject *list;
	unsigned int num_qubits;
	int verbose;
	if (!PyArg_ParseTuple(args, "IOp", &num_qubits, &list, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: gate_new(num_qubits, gate, verbose)");
		return NULL;
	}
	if (num_qubits == 0) {
		PyErr_SetString(DokiError, "num_qubits can't be zero");
		return NULL;
	}
	if (!PyList_Check(list)) {
		PyErr_SetString(DokiError, "gate must be a list of lists (matrix)");
		return NULL;
	}
	if (num_qubits > 30 || (Py_ssize_t)(1ull << num_qubits) != PyList_Size(list)) {
		PyErr_SetString(DokiError, "Wrong matrix size for specified number of qubits");
		return NULL;
	}
	const uint64_t dim = 1ull << num_qubits;
	if (num_qubits > 10) {
		PyErr_SetString(DokiError, "Failed to allocate qgate");
		return NULL;
	}
	double complex *m = (double complex *)malloc(sizeof(double complex) * dim * dim);
	if (!m) {
		PyErr_SetString(DokiError, "Failed to allocate qgate matrix");
		return NULL;
	}
	for (uint64_t i = 0; i < dim; i++) {
		PyObject *row = PyList_GetItem(list, (Py_ssize_t)i);
		if (!PyList_Check(row) || (uint64_t)PyList_Size(row) != dim) {
			free(m);
			PyErr_SetString(DokiError, "rows must be lists of size 2^num_qubits");
			return NULL;
		}
		for (uint64_t j = 0; j < dim; j++) {
			if (py_to_complex(PyList_GetItem(row, (Py_ssize_t)j), &m[i * dim + j])) {
				free(m);
				PyErr_SetString(DokiError, "matrix elements must be complex numbers");
				return NULL;
			}
		}
	}
	dk_gate *g = NULL;
	int rc = dk_gate_new(num_qubits, (const double *)m, &g);
	free(m);
	if (rc)
		return raise_dk(rc, "Failed to allocate qgate");
	PyObject *c = PyCapsule_New(g, CAP_GATE, gate_destroy);
	if (!c)
		dk_gate_free(g);
	return c;
}

static PyObject *doki_gate_get(PyObject *self, PyObject *args)
{
	PyObject *cap;
	int verbose;
	if (!PyArg_ParseTuple(args, "Op", &cap, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: gate_get(gate, verbose)");
		return NULL;
	}
	dk_gate *g = (dk_gate *)PyCapsule_GetPointer(cap, CAP_GATE);
	if (!g) {
		PyErr_SetString(DokiError, "NULL pointer to gate");
		return NULL;
	}
	const uint64_t dim = 1ull << dk_gate_num_qubits(g);
	double *m = (double *)malloc(16 * dim * dim);
	if (!m)
		return PyErr_NoMemory();
	dk_gate_get(g, m);
	PyObject *res = PyList_New((Py_ssize_t)dim);
	for (uint64_t i = 0; res && i < dim; i++) {
		PyObject *row = PyList_New((Py_ssize_t)dim);
		for (uint64_t j = 0; j < dim; j++)
			PyList_SET_ITEM(row, (Py_ssize_t)j,
					PyComplex_FromDoubles(m[2 * (i * dim + j)],
							      m[2 * (i * dim + j) + 1]));
		PyList_SET_ITEM(res, (Py_ssize_t)i, row);
	}
	free(m);
	return res;
}

/* ============================ registers ================================= */

static int check_precision(int p)
{
	if (p != DK_C64 && p != DK_C128) {
		PyErr_SetString(DokiError, "precision must be 1 (complex64) or 2 (complex128)");
		return -1;
	}
	return 0;
}

static PyObject *state_create_error(int rc)
{
	if (rc == DK_ERR_QUBITS)
		PyErr_SetString(DokiError, "Number of qubits exceeds maximum");
	else if (rc == DK_ERR_ALLOC || rc == DK_ERR_BUDGET)
		PyErr_SetString(DokiError, "Failed to allocate state vector");
	else
		return raise_dk(rc, "Unknown error when creating state");
	return NULL;
}

static PyObject *doki_registry_new(PyObject *self, PyObject *args)
{
	unsigned int num_qubits;
	int verbose, precision = DK_C128;
	if (!PyArg_ParseTuple(args, "Ip|i", &num_qubits, &verbose, &precision)) {
		PyErr_SetString(DokiError, "Syntax: registry_new(num_qubits, verbose)");
		return NULL;
	}
	if (num_qubits == 0) {
		PyErr_SetString(DokiError, "num_qubits can't be zero");
		return NULL;
	}
	if (check_precision(precision))
		return NULL;
	dk_state *s = NULL;
	int rc = dk_state_new(num_qubits, precision, &s);
	if (rc)
		return state_create_error(rc);
	return wrap_state(s);
}

static PyObject *doki_registry_new_data(PyObject *self, PyObject *args)
{
	PyObject *raw;
	unsigned int num_qubits;
	short verbose;
	int precision = DK_C128;
	if (!PyArg_ParseTuple(args, "IOh|i", &num_qubits, &raw, &verbose, &precision)) {
		PyErr_SetString(DokiError, "Syntax: registry_new_data(num_qubits, values, verbose)");
		return NULL;
	}
	if (num_qubits == 0) {
		PyErr_SetString(DokiError, "num_qubits can't be zero");
		return NULL;
	}
	if (check_precision(precision))
		return NULL;
	if (num_qubits > DK_MAX_QUBITS) {
		PyErr_SetString(DokiError, "Number of qubits exceeds maximum");
		return NULL;
	}
	const uint64_t size = 1ull << num_qubits;
	dk_state *s = NULL;
	int rc;
	if (PyObject_IsInstance(raw, np_ndarray) == 1) {
		PyObject *dt = PyObject_GetAttrString(raw, "dtype");
		PyObject *kind = dt ? PyObject_GetAttrString(dt, "kind") : NULL;
		Py_XDECREF(dt);
		const char *ks = kind ? PyUnicode_AsUTF8(kind) : NULL;
		int isnum = ks && strchr("biufc", ks[0]) != NULL;
		Py_XDECREF(kind);
		if (!isnum) {
			PyErr_SetString(DokiError, "values have to be numbers");
			return NULL;
		}
		PyObject *szo = PyObject_GetAttrString(raw, "size");
		Py_ssize_t sz = szo ? PyLong_AsSsize_t(szo) : -1;
		Py_XDECREF(szo);
		if ((uint64_t)sz != size) {
			PyErr_SetString(DokiError, "Wrong array size for the specified number of qubits");
			return NULL;
		}
		PyObject *flat = PyObject_CallMethod(raw, "ravel", NULL);
		PyObject *arr = flat ? PyObject_CallMethod(np_mod, "ascontiguousarray", "OO",
							   flat, np_complex128)
				     : NULL;
		Py_XDECREF(flat);
		if (!arr)
			return NULL;
		Py_buffer view;
		if (PyObject_GetBuffer(arr, &view, PyBUF_C_CONTIGUOUS) != 0) {
			Py_DECREF(arr);
			return NULL;
		}
		Py_BEGIN_ALLOW_THREADS rc = dk_state_from_host(num_qubits, precision,
							     (const double *)view.buf, &s);
		Py_END_ALLOW_THREADS PyBuffer_Release(&view);
		Py_DECREF(arr);
	} else if (PyList_Check(raw)) {
		if ((uint64_t)PyList_GET_SIZE(raw) != size) {
			PyErr_SetString(DokiError,
					"Wrong list size for the specified number of qubits\n");
			return NULL;
		}
		double *h = (double *)malloc(16 * size);
		if (!h)
			return PyErr_NoMemory();
		for (uint64_t i = 0; i < size; i++) {
			Py_complex z = PyComplex_AsCComplex(PyList_GET_ITEM(raw, (Py_ssize_t)i));
			if (z.real == -1.0 && PyErr_Occurred()) {
				free(h);
				PyErr_Clear();
				PyErr_SetString(DokiError, "values have to be numbers");
				return NULL;
			}
			h[2 * i] = z.real;
			h[2 * i + 1] = z.imag;
		}
		rc = dk_state_from_host(num_qubits, precision, h, &s);
		free(h);
	} else {
		PyErr_SetString(DokiError, "values has to be either a python list or a numpy array");
		return NULL;
	}
	if (rc)
		return state_create_error(rc);
	return wrap_state(s);
}

static int check_threads(int t)
{
	if (t <= 0 && t != -1) {
		PyErr_SetString(DokiError, THREADS_MSG);
		return -1;
	}
	return 0;
}

static PyObject *doki_registry_clone(PyObject *self, PyObject *args)
{
	PyObject *cap;
	int num_threads, verbose;
	if (!PyArg_ParseTuple(args, "Oip", &cap, &num_threads, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: registry_clone(registry, num_threads, verbose)");
		return NULL;
	}
	if (check_threads(num_threads))
		return NULL;
	dk_state *src = get_state(cap, "NULL pointer to source registry");
	if (!src)
		return NULL;
	dk_state *s = NULL;
	int rc = dk_state_clone(src, &s);
	if (rc)
		return raise_dk(rc, "Unknown error when cloning state");
	return wrap_state(s);
}

static PyObject *doki_registry_del(PyObject *self, PyObject *args)
{
	PyObject *cap;
	int verbose;
	if (!PyArg_ParseTuple(args, "Op", &cap, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: registry_del(registry, verbose)");
		return NULL;
	}
	dk_state *s = (dk_state *)PyCapsule_GetPointer(cap, CAP_STATE);
	if (s)
		dk_state_release(s);
	else
		PyErr_Clear();
	Py_RETURN_NONE;
}

static PyObject *doki_registry_get(PyObject *self, PyObject *args)
{
	PyObject *cap;
	unsigned long long id;
	int canonical, verbose;
	if (!PyArg_ParseTuple(args, "OKpp", &cap, &id, &canonical, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: registry_get(registry, id, canonical, verbose)");
		return NULL;
	}
	dk_state *s = get_state(cap, "NULL pointer to registry");
	if (!s)
		return NULL;
	if (dk_state_num_qubits(s) < 64 && id >= (1ull << dk_state_num_qubits(s))) {
		PyErr_SetString(DokiError, "Index out of range");
		return NULL;
	}
	double re, im;
	int rc;
	Py_BEGIN_ALLOW_THREADS rc = dk_get_amplitude(s, id, &re, &im);
	Py_END_ALLOW_THREADS if (rc) return raise_dk(rc, "Failed to read registry");
	double complex val = re + I * im;
	if (canonical) {
		double phase;
		Py_BEGIN_ALLOW_THREADS rc = dk_global_phase(s, &phase);
		Py_END_ALLOW_THREADS if (rc) return raise_dk(rc, "Failed to read registry");
		val = val * (cos(phase) - I * sin(phase));
	}
	return PyComplex_FromDoubles(creal(val), cimag(val));
}

static PyObject *doki_registry_get_all(PyObject *self, PyObject *args)
{
	PyObject *cap;
	int canonical = 0;
	if (!PyArg_ParseTuple(args, "O|p", &cap, &canonical)) {
		PyErr_SetString(DokiError, "Syntax: registry_get_all(registry, canonical)");
		return NULL;
	}
	dk_state *s = get_state(cap, "NULL pointer to registry");
	if (!s)
		return NULL;
	const uint64_t size = 1ull << dk_state_num_qubits(s);
	PyObject *arr = PyObject_CallMethod(np_mod, "empty", "KO", (unsigned long long)size,
					    np_complex128);
	if (!arr)
		return NULL;
	Py_buffer view;
	if (PyObject_GetBuffer(arr, &view, PyBUF_C_CONTIGUOUS | PyBUF_WRITABLE) != 0) {
		Py_DECREF(arr);
		return NULL;
	}
	int rc;
	double phase = 0.0;
	Py_BEGIN_ALLOW_THREADS rc = dk_get_amplitudes(s, 0, size, (double *)view.buf);
	if (!rc && canonical)
		rc = dk_global_phase(s, &phase);
	Py_END_ALLOW_THREADS if (rc)
	{
		PyBuffer_Release(&view);
		Py_DECREF(arr);
		return raise_dk(rc, "Failed to read registry");
	}
	if (canonical) {
		double complex *v = (double complex *)view.buf;
		const double complex f = cos(phase) - I * sin(phase);
		for (uint64_t i = 0; i < size; i++)
			v[i] = v[i] * f;
	}
	PyBuffer_Release(&view);
	return arr;
}

static int parse_qubit_set(PyObject *set, unsigned n, unsigned *out, unsigned count,
			   const char *type_msg, const char *range_msg,
			   PyObject *forbid, const char *forbid_msg)
{
	PyObject *copy = PySet_New(set);
	if (!copy)
		return -1;
	for (unsigned i = 0; i < count; i++) {
		PyObject *v = PySet_Pop(copy);
		if (!v || !PyLong_Check(v)) {
			Py_XDECREF(v);
			Py_DECREF(copy);
			PyErr_SetString(DokiError, type_msg);
			return -1;
		}
		if (forbid && PySet_Contains(forbid, v)) {
			/* the reference tests membership in the control set even when it is
			 * None (PySet_Contains then fails, which it treats as true) */
			Py_DECREF(v);
			Py_DECREF(copy);
			PyErr_Clear();
			PyErr_SetString(DokiError, forbid_msg);
			return -1;
		}
		long q = PyLong_AsLong(v);
		Py_DECREF(v);
		if (q < 0 || (unsigned long)q >= n) {
			Py_DECREF(copy);
			PyErr_Clear();
			PyErr_SetString(DokiError, range_msg);
			return -1;
		}
		out[i] = (unsigned)q;
	}
	Py_DECREF(copy);
	return 0;
}

static PyObject *doki_registry_apply(PyObject *self, PyObject *args)
{
	PyObject *scap, *gcap, *tlist, *cset, *aset;
	int num_threads, verbose;
	if (!PyArg_ParseTuple(args, "OOOOOip", &scap, &gcap, &tlist, &cset, &aset,
			      &num_threads, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: registry_apply(registry, gate, target_list, "
					   "control_set, anticontrol_set, num_threads, verbose)");
		return NULL;
	}
	if (check_threads(num_threads))
		return NULL;
	dk_state *s = get_state(scap, "NULL pointer to registry");
	if (!s)
		return NULL;
	dk_gate *g = (dk_gate *)PyCapsule_GetPointer(gcap, CAP_GATE);
	if (!g) {
		PyErr_SetString(DokiError, "NULL pointer to gate");
		return NULL;
	}
	if (!PyList_Check(tlist)) {
		PyErr_SetString(DokiError, "target_list must be a list");
		return NULL;
	}
	const unsigned nt = (unsigned)PyList_Size(tlist);
	if (nt != dk_gate_num_qubits(g)) {
		PyErr_SetString(DokiError, "Wrong number of targets specified for that gate");
		return NULL;
	}
	unsigned nc = 0, na = 0;
	if (PySet_Check(cset))
		nc = (unsigned)PySet_Size(cset);
	else if (cset != Py_None) {
		PyErr_SetString(DokiError, "control_set must be a set or None");
		return NULL;
	}
	if (PySet_Check(aset))
		na = (unsigned)PySet_Size(aset);
	else if (aset != Py_None) {
		PyErr_SetString(DokiError, "anticontrol_set must be a set or None");
		return NULL;
	}
	const unsigned n = dk_state_num_qubits(s);
	unsigned tg[16], *ctl = NULL, *act = NULL;
	ctl = (unsigned *)malloc(sizeof(unsigned) * (nc + 1));
	act = (unsigned *)malloc(sizeof(unsigned) * (na + 1));
	if (!ctl || !act) {
		free(ctl);
		free(act);
		return PyErr_NoMemory();
	}
	PyObject *res = NULL;
	if (nc > 0 && parse_qubit_set(cset, n, ctl, nc,
				      "control_set must be a set qubit ids (unsigned integers)",
				      "Control qubit out of range", NULL, NULL))
		goto done;
	if (na > 0 && parse_qubit_set(aset, n, act, na,
				      "anticontrol_set must be a set qubit ids (unsigned integers)",
				      "Anticontrol qubit out of range", cset,
				      "A control cannot also be an anticontrol"))
		goto done;
	for (unsigned i = 0; i < nt; i++) {
		PyObject *v = PyList_GetItem(tlist, (Py_ssize_t)i);
		if (!PyLong_Check(v)) {
			PyErr_SetString(DokiError,
					"target_list must be a list of qubit ids (unsigned integers)");
			goto done;
		}
		if ((nc > 0 && PySet_Contains(cset, v)) || (na > 0 && PySet_Contains(aset, v))) {
			PyErr_SetString(DokiError, "A target cannot also be a control or an anticontrol");
			goto done;
		}
		long q = PyLong_AsLong(v);
		if (q < 0 || (unsigned long)q >= n) {
			PyErr_Clear();
			PyErr_SetString(DokiError, "Target qubit out of range");
			goto done;
		}
		for (unsigned j = 0; j < i; j++)
			if (tg[j] == (unsigned)q) {
				PyErr_SetString(DokiError, "Repeated target qubit");
				goto done;
			}
		tg[i] = (unsigned)q;
	}
	{
		dk_state *out = NULL;
		int rc = dk_apply_gate(s, g, tg, nt, ctl, nc, act, na, &out);
		if (rc == DK_ERR_ALLOC || rc == DK_ERR_BUDGET)
			PyErr_SetString(DokiError, "Failed to allocate new state chunk");
		else if (rc)
			raise_dk(rc, "Unknown error when applying gate");
		else
			res = wrap_state(out);
	}
done:
	free(ctl);
	free(act);
	return res;
}

/* A C-contiguous buffer of `count` items of `itemsize` bytes (count < 0:
 * any length; the length is returned through *len). */
static int get_array(PyObject *obj, Py_buffer *view, Py_ssize_t itemsize, Py_ssize_t count,
		     Py_ssize_t *len, const char *name)
{
	if (PyObject_GetBuffer(obj, view, PyBUF_C_CONTIGUOUS | PyBUF_FORMAT) != 0) {
		PyErr_Clear();
		PyErr_Format(DokiError, "%s must be a contiguous numpy array", name);
		return -1;
	}
	if (view->itemsize != itemsize || (count >= 0 && view->len != count * itemsize)) {
		PyBuffer_Release(view);
		PyErr_Format(DokiError, "%s has the wrong item size or length", name);
		return -1;
	}
	if (len)
		*len = view->len / itemsize;
	return 0;
}

/* registry_apply_many(registry, op_k, op_targets, op_controls, op_anticontrols,
 * op_matrix, matrices): every gate of a circuit in one call (the serving
 * form's submission path; the reference applies one gate per
 * registry_apply call, doki.c:722-941).  Arrays as dk_apply_gates takes
 * them: uint32 op_k [N], uint32 op_targets [N, 3], uint64 op_controls [N],
 * uint64 op_anticontrols [N], uint64 op_matrix [N], complex128 matrices. */
static PyObject *doki_registry_apply_many(PyObject *self, PyObject *args)
{
	PyObject *scap, *ok, *ot, *oc, *oa, *om, *mats;
	if (!PyArg_ParseTuple(args, "OOOOOOO", &scap, &ok, &ot, &oc, &oa, &om, &mats)) {
		PyErr_SetString(DokiError, "Syntax: registry_apply_many(registry, op_k, op_targets, "
					   "op_controls, op_anticontrols, op_matrix, matrices)");
		return NULL;
	}
	dk_state *s = get_state(scap, "NULL pointer to registry");
	if (!s)
		return NULL;
	Py_buffer vk, vt, vc, va, vm, vx;
	Py_ssize_t n = 0, nm = 0;
	if (get_array(ok, &vk, 4, -1, &n, "op_k"))
		return NULL;
	PyObject *res = NULL;
	int got = 1;
	if (get_array(ot, &vt, 4, 3 * n, NULL, "op_targets"))
		goto r1;
	got++;
	if (get_array(oc, &vc, 8, n, NULL, "op_controls"))
		goto r2;
	got++;
	if (get_array(oa, &va, 8, n, NULL, "op_anticontrols"))
		goto r3;
	got++;
	if (get_array(om, &vm, 8, n, NULL, "op_matrix"))
		goto r4;
	got++;
	if (get_array(mats, &vx, 16, -1, &nm, "matrices"))
		goto r5;
	{
		dk_state *out = NULL;
		int rc;
		Py_BEGIN_ALLOW_THREADS rc = dk_apply_gates(
			s, (unsigned)n, (const unsigned *)vk.buf, (const unsigned *)vt.buf,
			(const uint64_t *)vc.buf, (const uint64_t *)va.buf, (const uint64_t *)vm.buf,
			(const double *)vx.buf, (uint64_t)nm, &out);
		Py_END_ALLOW_THREADS if (rc) raise_dk(rc, "Failed to apply the gates");
		else res = wrap_state(out);
	}
	PyBuffer_Release(&vx);
r5:
	PyBuffer_Release(&vm);
r4:
	PyBuffer_Release(&va);
r3:
	PyBuffer_Release(&vc);
r2:
	PyBuffer_Release(&vt);
r1:
	PyBuffer_Release(&vk);
	(void)got;
	return res;
}

/* Distributed registers' local view (dk_state_norm / read_half /
 * replace_half): pointers are integers (numpy .ctypes.data, a torch
 * tensor's data_ptr()), in the register's storage precision. */
static PyObject *doki_registry_norm(PyObject *self, PyObject *args)
{
	PyObject *cap;
	if (!PyArg_ParseTuple(args, "O", &cap)) {
		PyErr_SetString(DokiError, "Syntax: registry_norm(registry)");
		return NULL;
	}
	dk_state *s = get_state(cap, "NULL pointer to registry");
	if (!s)
		return NULL;
	double nrm = 0.0, stored = 0.0;
	int rc;
	Py_BEGIN_ALLOW_THREADS rc = dk_state_norm(s, &nrm, &stored);
	Py_END_ALLOW_THREADS if (rc) return raise_dk(rc, "Failed to read the norm");
	return Py_BuildValue("(dd)", nrm, stored);
}

static PyObject *doki_registry_read_half(PyObject *self, PyObject *args)
{
	PyObject *cap;
	unsigned bit;
	int value, on_device;
	double scale;
	unsigned long long ptr;
	if (!PyArg_ParseTuple(args, "OIidKp", &cap, &bit, &value, &scale, &ptr, &on_device)) {
		PyErr_SetString(DokiError, "Syntax: registry_read_half(registry, bit, value, scale, "
					   "dst_pointer, on_device)");
		return NULL;
	}
	dk_state *s = get_state(cap, "NULL pointer to registry");
	if (!s)
		return NULL;
	int rc;
	Py_BEGIN_ALLOW_THREADS rc = dk_state_read_half(s, bit, value, scale, (void *)ptr, on_device);
	Py_END_ALLOW_THREADS if (rc) return raise_dk(rc, "Failed to read half of the registry");
	Py_RETURN_NONE;
}

static PyObject *doki_registry_replace_half(PyObject *self, PyObject *args)
{
	PyObject *cap;
	unsigned bit;
	int value, on_device;
	double scale;
	unsigned long long ptr;
	if (!PyArg_ParseTuple(args, "OIidKp", &cap, &bit, &value, &scale, &ptr, &on_device)) {
		PyErr_SetString(DokiError, "Syntax: registry_replace_half(registry, bit, value, "
					   "scale, src_pointer, on_device)");
		return NULL;
	}
	dk_state *s = get_state(cap, "NULL pointer to registry");
	if (!s)
		return NULL;
	dk_state *out = NULL;
	int rc;
	Py_BEGIN_ALLOW_THREADS rc = dk_state_replace_half(s, bit, value, scale, (const void *)ptr,
							   on_device, &out);
	Py_END_ALLOW_THREADS if (rc) return raise_dk(rc, "Failed to replace half of the registry");
	return wrap_state(out);
}

static PyObject *doki_registry_join(PyObject *self, PyObject *args)
{
	PyObject *c1, *c2;
	int num_threads, verbose;
	if (!PyArg_ParseTuple(args, "OOip", &c1, &c2, &num_threads, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: registry_join(most_registry, "
					   "least_registry, num_threads, verbose)");
		return NULL;
	}
	if (check_threads(num_threads))
		return NULL;
	dk_state *a = get_state(c1, "NULL pointer to registry1");
	if (!a)
		return NULL;
	dk_state *b = get_state(c2, "NULL pointer to registry2");
	if (!b)
		return NULL;
	dk_state *out = NULL;
	int rc;
	Py_BEGIN_ALLOW_THREADS rc = dk_join(a, b, &out);
	Py_END_ALLOW_THREADS if (rc == DK_ERR_ALLOC || rc == DK_ERR_BUDGET)
	{
		PyErr_SetString(DokiError, "Failed to allocate new state chunk");
		return NULL;
	}
	if (rc)
		return raise_dk(rc, "Unknown error when joining states");
	return wrap_state(out);
}

static PyObject *doki_registry_measure(PyObject *self, PyObject *args)
{
	PyObject *cap, *rolls;
	unsigned long long mask;
	int num_threads, verbose;
	if (!PyArg_ParseTuple(args, "OKOip", &cap, &mask, &rolls, &num_threads, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: registry_measure(registry, mask, "
					   "roll_list, num_threads, verbose)");
		return NULL;
	}
	if (check_threads(num_threads))
		return NULL;
	dk_state *s = get_state(cap, "NULL pointer to registry");
	if (!s)
		return NULL;
	if (!PyList_Check(rolls)) {
		PyErr_SetString(DokiError, "roll_list must be a list of real numbers in [0, 1)!");
		return NULL;
	}
	const unsigned n = dk_state_num_qubits(s);
	/* doki.c:1097-1121: one roll per measured qubit, highest qubit first */
	unsigned need = 0;
	for (unsigned q = 0; q < n && q < 64; q++)
		if ((mask >> q) & 1ull)
			need++;
	double *rv = (double *)malloc(sizeof(double) * (need + 1));
	int8_t *res = (int8_t *)malloc(n + 1);
	if (!rv || !res) {
		free(rv);
		free(res);
		return PyErr_NoMemory();
	}
	for (unsigned i = 0; i < need; i++) {
		double r = -1.0;
		if ((Py_ssize_t)i < PyList_Size(rolls)) {
			r = PyFloat_AsDouble(PyList_GetItem(rolls, (Py_ssize_t)i));
			if (r == -1.0 && PyErr_Occurred())
				PyErr_Clear();
		}
		if (r < 0 || r >= 1) {
			free(rv);
			free(res);
			PyErr_SetString(DokiError, "roll not in interval [0, 1)!");
			return NULL;
		}
		rv[i] = r;
	}
	dk_state *out = NULL;
	int rc;
	Py_BEGIN_ALLOW_THREADS rc = dk_measure_mask(s, mask, rv, need, res, &out);
	Py_END_ALLOW_THREADS free(rv);
	if (rc) {
		free(res);
		if (rc == DK_ERR_NORM0) {
			PyErr_SetString(DokiError, "New normalization constant is 0. Please report "
						   "this error with the steps to reproduce it.");
			return NULL;
		}
		if (rc == DK_ERR_ALLOC || rc == DK_ERR_BUDGET) {
			PyErr_SetString(DokiError, "Failed to allocate state vector");
			return NULL;
		}
		return raise_dk(rc, "Unknown error while collapsing state");
	}
	PyObject *lst = PyList_New(n);
	for (unsigned i = 0; i < n; i++) {
		PyObject *v = res[i] < 0 ? Py_None : (res[i] ? Py_True : Py_False);
		Py_INCREF(v);
		PyList_SET_ITEM(lst, i, v);
	}
	free(res);
	PyObject *rc_obj;
	if (out)
		rc_obj = wrap_state(out);
	else {
		rc_obj = Py_None;
		Py_INCREF(rc_obj);
	}
	PyObject *tup = PyTuple_Pack(2, rc_obj, lst);
	Py_DECREF(rc_obj);
	Py_DECREF(lst);
	return tup;
}

static PyObject *doki_registry_prob(PyObject *self, PyObject *args)
{
	PyObject *cap;
	unsigned int id;
	int num_threads, verbose;
	if (!PyArg_ParseTuple(args, "OIip", &cap, &id, &num_threads, &verbose)) {
		PyErr_SetString(DokiError,
				"Syntax: registry_prob(registry, qubit_id, num_threads, verbose)");
		return NULL;
	}
	if (check_threads(num_threads))
		return NULL;
	dk_state *s = get_state(cap, "NULL pointer to registry");
	if (!s)
		return NULL;
	if (id >= dk_state_num_qubits(s)) {
		PyErr_SetString(DokiError, "Qubit id out of range");
		return NULL;
	}
	double p;
	int rc;
	Py_BEGIN_ALLOW_THREADS rc = dk_probability(s, id, &p);
	Py_END_ALLOW_THREADS if (rc) return raise_dk(rc, "Failed to compute probability");
	return PyFloat_FromDouble(p);
}

static PyObject *doki_registry_probs(PyObject *self, PyObject *args)
{
	PyObject *cap;
	if (!PyArg_ParseTuple(args, "O", &cap)) {
		PyErr_SetString(DokiError, "Syntax: registry_probs(registry)");
		return NULL;
	}
	dk_state *s = get_state(cap, "NULL pointer to registry");
	if (!s)
		return NULL;
	const unsigned n = dk_state_num_qubits(s);
	double p[64];
	int rc;
	Py_BEGIN_ALLOW_THREADS rc = dk_marginals(s, p);
	Py_END_ALLOW_THREADS if (rc) return raise_dk(rc, "Failed to compute probabilities");
	PyObject *lst = PyList_New(n);
	for (unsigned q = 0; q < n; q++)
		PyList_SET_ITEM(lst, q, PyFloat_FromDouble(p[q]));
	return lst;
}

static PyObject *doki_registry_density(PyObject *self, PyObject *args)
{
	PyObject *cap;
	int verbose;
	if (!PyArg_ParseTuple(args, "Op", &cap, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: registry_density(state, verbose)");
		return NULL;
	}
	dk_state *s = get_state(cap, "NULL pointer to registry");
	if (!s)
		return NULL;
	const unsigned n = dk_state_num_qubits(s);
	fmat *m = fmat_new(FM_DENSITY, 1ull << n, 1ull << n);
	if (!m) {
		PyErr_SetString(DokiError, "[DENSITY] Failed to allocate density matrix");
		return NULL;
	}
	Py_INCREF(cap);
	m->a = cap;
	return wrap_fmat(m);
}

static PyObject *doki_registry_mem(PyObject *self, PyObject *args)
{
	PyObject *cap;
	int verbose;
	if (!PyArg_ParseTuple(args, "Op", &cap, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: registry_mem(state, verbose)");
		return NULL;
	}
	dk_state *s = get_state(cap, "NULL pointer to registry");
	if (!s)
		return NULL;
	return PyLong_FromSize_t(dk_state_mem_size(s));
}

static PyObject *doki_registry_precision(PyObject *self, PyObject *args)
{
	PyObject *cap;
	if (!PyArg_ParseTuple(args, "O", &cap))
		return NULL;
	dk_state *s = get_state(cap, "NULL pointer to registry");
	if (!s)
		return NULL;
	return PyLong_FromLong(dk_state_precision(s));
}

static PyObject *doki_engine_sync(PyObject *self, PyObject *args)
{
	int rc;
	Py_BEGIN_ALLOW_THREADS rc = dk_sync();
	Py_END_ALLOW_THREADS if (rc) return raise_dk(rc, "sync failed");
	Py_RETURN_NONE;
}

static PyObject *doki_engine_set_fusion(PyObject *self, PyObject *args)
{
	int enable;
	if (!PyArg_ParseTuple(args, "p", &enable))
		return NULL;
	dk_set_fusion(enable);
	Py_RETURN_NONE;
}

static PyObject *doki_engine_stats(PyObject *self, PyObject *args)
{
	uint64_t l = 0, s = 0, g = 0, hi = 0, ho = 0, me = 0, tp = 0, te = 0;
	dk_get_stats(&l, &s, &g);
	dk_get_io_stats(&hi, &ho);
	dk_get_mma_stats(&me);
	dk_get_tm_stats(&tp, &te);
	return Py_BuildValue("{s:K,s:K,s:K,s:K,s:K,s:K,s:K,s:K}", "kernel_launches",
			     (unsigned long long)l, "sweeps", (unsigned long long)s, "gates",
			     (unsigned long long)g, "h2d_bytes", (unsigned long long)hi,
			     "d2h_bytes", (unsigned long long)ho, "mma_entry_amplitudes",
			     (unsigned long long)me, "tm_sweeps_presplit", (unsigned long long)tp,
			     "tm_sweeps_entry_b", (unsigned long long)te);
}

static PyObject *doki_registry_compare(PyObject *self, PyObject *args)
{
	PyObject *c1, *c2;
	if (!PyArg_ParseTuple(args, "OO", &c1, &c2)) {
		PyErr_SetString(DokiError, "Syntax: registry_compare(registry1, registry2)");
		return NULL;
	}
	dk_state *a = get_state(c1, "NULL pointer to registry1");
	if (!a)
		return NULL;
	dk_state *b = get_state(c2, "NULL pointer to registry2");
	if (!b)
		return NULL;
	double fid = 0.0, err = 0.0;
	int rc;
	Py_BEGIN_ALLOW_THREADS rc = dk_compare_states(a, b, &fid, &err);
	Py_END_ALLOW_THREADS if (rc) return raise_dk(rc, "Failed to compare registries");
	return Py_BuildValue("(dd)", fid, err);
}

static PyObject *doki_engine_new_slot(PyObject *self, PyObject *args)
{
	int slot = -1, rc;
	Py_BEGIN_ALLOW_THREADS rc = dk_slot_new(&slot);
	Py_END_ALLOW_THREADS if (rc) return raise_dk(rc, "Failed to create a stream slot");
	return PyLong_FromLong(slot);
}

static PyObject *doki_engine_set_slot(PyObject *self, PyObject *args)
{
	int slot;
	if (!PyArg_ParseTuple(args, "i", &slot))
		return NULL;
	int rc = dk_slot_set(slot);
	if (rc)
		return raise_dk(rc, "Failed to select the stream slot");
	Py_RETURN_NONE;
}

static PyObject *doki_engine_get_slot(PyObject *self, PyObject *args)
{
	return PyLong_FromLong(dk_slot_get());
}

static PyObject *doki_engine_stream(PyObject *self, PyObject *args)
{
	return PyLong_FromVoidPtr(dk_stream());
}

static PyObject *doki_registry_flush(PyObject *self, PyObject *args)
{
	PyObject *cap;
	if (!PyArg_ParseTuple(args, "O", &cap)) {
		PyErr_SetString(DokiError, "Syntax: registry_flush(registry)");
		return NULL;
	}
	dk_state *s = get_state(cap, "NULL pointer to registry");
	if (!s)
		return NULL;
	int rc;
	Py_BEGIN_ALLOW_THREADS rc = dk_state_flush(s);
	Py_END_ALLOW_THREADS if (rc) return raise_dk(rc, "Failed to apply queued gates");
	Py_RETURN_NONE;
}

/* ===================== functional-matrix API ============================ */

static fmat *get_fmat(PyObject *cap)
{
	fmat *m = (fmat *)PyCapsule_GetPointer(cap, CAP_FMAT);
	if (!m)
		PyErr_SetString(DokiError, "NULL pointer to matrix");
	return m;
}

/* The reference raises DokiError over the capsule's own error. */
static fmat *get_fmat_msg(PyObject *cap, const char *msg)
{
	fmat *m = (fmat *)PyCapsule_GetPointer(cap, CAP_FMAT);
	if (!m) {
		PyErr_Clear();
		PyErr_SetString(DokiError, msg);
	}
	return m;
}

static PyObject *doki_funmatrix_create(PyObject *self, PyObject *args)
{
	PyObject *list;
	int verbose;
	if (!PyArg_ParseTuple(args, "Op", &list, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: funmatrix_create(matrix, verbose)");
		return NULL;
	}
	if (!PyList_Check(list)) {
		PyErr_SetString(DokiError, "matrix must be a list of lists (matrix)");
		return NULL;
	}
	Py_ssize_t nr = PyList_Size(list);
	if (nr == 0) {
		PyErr_SetString(DokiError, "there are no rows");
		return NULL;
	}
	PyObject *row = PyList_GetItem(list, 0);
	if (!PyList_Check(row)) {
		PyErr_SetString(DokiError, "rows must be lists");
		return NULL;
	}
	Py_ssize_t nc = PyList_Size(row);
	if (nc == 0) {
		PyErr_SetString(DokiError, "there are no columns");
		return NULL;
	}
	fmat *m = fmat_new(FM_CUSTOM, (uint64_t)nr, (uint64_t)nc);
	fm_buf *d = (fm_buf *)malloc(sizeof(fm_buf) + sizeof(double complex) * nr * nc);
	if (!m || !d) {
		free(m);
		free(d);
		PyErr_SetString(DokiError, "failed to allocate 2D matrix");
		return NULL;
	}
	d->refs = 1;
	d->len = (size_t)(nr * nc);
	m->data = d;
	for (Py_ssize_t i = 0; i < nr; i++) {
		row = PyList_GetItem(list, i);
		if (!PyList_Check(row) || PyList_Size(row) != nc) {
			fmat_free(m);
			PyErr_SetString(DokiError, "rows must be lists of the same size");
			return NULL;
		}
		for (Py_ssize_t j = 0; j < nc; j++)
			if (py_to_complex(PyList_GetItem(row, j), &d->v[i * nc + j])) {
				fmat_free(m);
				PyErr_SetString(DokiError, "matrix elements must be complex numbers");
				return NULL;
			}
	}
	return wrap_fmat(m);
}

static PyObject *fm_simple(PyObject *args, const char *syntax, int kind, int vector)
{
	unsigned int n;
	int verbose;
	if (!PyArg_ParseTuple(args, "Ip", &n, &verbose)) {
		PyErr_SetString(DokiError, syntax);
		return NULL;
	}
	if (n > 62) {
		PyErr_SetString(DokiError, "Number of qubits exceeds maximum");
		return NULL;
	}
	fmat *m = fmat_new(kind, 1ull << n, vector ? 1 : (1ull << n));
	if (!m) {
		PyErr_SetString(DokiError, "NULL pointer to matrix");
		return NULL;
	}
	return wrap_fmat(m);
}

static PyObject *doki_funmatrix_identity(PyObject *self, PyObject *args)
{
	return fm_simple(args, "Syntax: funmatrix_identity(num_qubits, verbose)", FM_IDENTITY, 0);
}

static PyObject *doki_funmatrix_statezero(PyObject *self, PyObject *args)
{
	return fm_simple(args, "Syntax: funmatrix_statezero(num_qubits, verbose)", FM_STATEZERO, 1);
}

static PyObject *doki_funmatrix_densityzero(PyObject *self, PyObject *args)
{
	return fm_simple(args, "Syntax: funmatrix_densityzero(num_qubits, verbose)",
			 FM_DENSITYZERO, 0);
}

static PyObject *doki_funmatrix_hadamard(PyObject *self, PyObject *args)
{
	PyObject *r = fm_simple(args, "Syntax: funmatrix_hadamard(num_qubits, verbose)", FM_WALSH, 0);
	if (r) {
		fmat *m = (fmat *)PyCapsule_GetPointer(r, CAP_FMAT);
		m->hadamard = 1;
	}
	return r;
}

static PyObject *doki_funmatrix_addcontrol(PyObject *self, PyObject *args)
{
	PyObject *cap;
	int verbose;
	if (!PyArg_ParseTuple(args, "Op", &cap, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: funmatrix_addcontrol(funmatrix, verbose)");
		return NULL;
	}
	fmat *u = get_fmat_msg(cap, "NULL pointer to matrix");
	if (!u)
		return NULL;
	fmat *m = fmat_new(FM_CU, u->r * 2, u->c * 2);
	if (!m) {
		PyErr_SetString(DokiError, "NULL pointer to matrix");
		return NULL;
	}
	Py_INCREF(cap);
	m->a = cap;
	return wrap_fmat(m);
}

/* Reference getitem codes -> its messages (doki.c:1528-1570, 2155-2205). */
static PyObject *get_error(int rc, const char *prefix)
{
	static const char *const what[] = {
		"Error adding parent matrices",
		"Error substracting parent matrices",
		"Error multiplying parent matrices",
		"Error multiplying entity-wise parent matrices",
		"Error calculating Kronecker product of parent matrices",
		"Unknown operation between parent matrices",
		"Element out of bounds",
		"f returned NAN",
	};
	if (rc >= FMG_ADD && rc <= FMG_NAN)
		PyErr_Format(DokiError, "[%s] %s", prefix, what[rc - FMG_ADD]);
	else if (rc == DK_ERR_ARG)
		PyErr_Format(DokiError, "[%s] Element out of bounds", prefix);
	else
		raise_dk(rc, prefix);
	return NULL;
}

static PyObject *doki_funmatrix_get(PyObject *self, PyObject *args)
{
	PyObject *cap;
	unsigned long long i, j;
	int verbose;
	if (!PyArg_ParseTuple(args, "OKKp", &cap, &i, &j, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: funmatrix_get(funmatrix, i, j, verbose)");
		return NULL;
	}
	fmat *m = get_fmat_msg(cap, "NULL pointer to matrix");
	if (!m)
		return NULL;
	if (i >= m->r || j >= m->c) {
		PyErr_SetString(DokiError, "Out of bounds");
		return NULL;
	}
	double complex v;
	int rc = fmat_get(m, i, j, &v);
	if (rc)
		return get_error(rc, "GET");
	if (isnan(creal(v)) || isnan(cimag(v))) {
		PyErr_SetString(DokiError, "[GET] Unexpected NAN value");
		return NULL;
	}
	return PyComplex_FromDoubles(creal(v), cimag(v));
}

static PyObject *doki_funmatrix_numpy(PyObject *self, PyObject *args)
{
	PyObject *cap;
	if (!PyArg_ParseTuple(args, "O", &cap)) {
		PyErr_SetString(DokiError, "Syntax: funmatrix_numpy(funmatrix)");
		return NULL;
	}
	fmat *m = get_fmat(cap);
	if (!m)
		return NULL;
	if (m->r == 0 || m->c == 0 || m->r > (1ull << 28) || m->c > (1ull << 28) ||
	    m->r * m->c > (1ull << 28)) {
		PyErr_SetString(DokiError, "matrix too large to export");
		return NULL;
	}
	/* make sure a reduced density matrix is materialised in one call */
	double complex first;
	int rc = fmat_get(m, 0, 0, &first);
	if (rc)
		return get_error(rc, "GET");
	PyObject *shape = Py_BuildValue("(KK)", (unsigned long long)m->r, (unsigned long long)m->c);
	PyObject *arr = PyObject_CallMethod(np_mod, "empty", "OO", shape, np_complex128);
	Py_DECREF(shape);
	if (!arr)
		return NULL;
	Py_buffer view;
	if (PyObject_GetBuffer(arr, &view, PyBUF_C_CONTIGUOUS | PyBUF_WRITABLE) != 0) {
		Py_DECREF(arr);
		return NULL;
	}
	double complex *out = (double complex *)view.buf;
	if (m->kind == FM_PTRACE && m->mat_ready && fmat_plain(m))
		memcpy(out, m->rho, sizeof(double complex) * m->r * m->c);
	else if (m->kind == FM_CUSTOM && fmat_plain(m))
		memcpy(out, m->data->v, sizeof(double complex) * m->r * m->c);
	else {
		for (uint64_t i = 0; i < m->r && !rc; i++)
			for (uint64_t j = 0; j < m->c && !rc; j++)
				rc = fmat_get(m, i, j, &out[i * m->c + j]);
	}
	PyBuffer_Release(&view);
	if (rc) {
		Py_DECREF(arr);
		return get_error(rc, "GET");
	}
	return arr;
}

static PyObject *doki_funmatrix_shape(PyObject *self, PyObject *args)
{
	PyObject *cap;
	int verbose;
	if (!PyArg_ParseTuple(args, "Op", &cap, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: funmatrix_shape(funmatrix, verbose)");
		return NULL;
	}
	fmat *m = get_fmat_msg(cap, "NULL pointer to matrix");
	if (!m)
		return NULL;
	return Py_BuildValue("(KK)", (unsigned long long)m->r, (unsigned long long)m->c);
}

static PyObject *doki_funmatrix_partialtrace(PyObject *self, PyObject *args)
{
	PyObject *cap;
	unsigned int id;
	int verbose;
	if (!PyArg_ParseTuple(args, "OIp", &cap, &id, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: funmatrix_partialtrace(funmatrix, id, verbose)");
		return NULL;
	}
	fmat *p = get_fmat_msg(cap, "[PTRACE] The matrix is NULL");
	if (!p)
		return NULL;
	if (p->r != p->c) {
		PyErr_SetString(DokiError, "[PTRACE] The matrix is not a square matrix");
		return NULL;
	}
	if ((int)id < 0) {
		PyErr_SetString(DokiError, "[PTRACE] elem id has to be >= 0");
		return NULL;
	}
	if ((int)id >= ilog2(p->r)) {
		PyErr_SetString(DokiError, "[PTRACE] elem id out of range");
		return NULL;
	}
	fmat *m = fmat_new(FM_PTRACE, p->r >> 1, p->c >> 1);
	if (!m) {
		PyErr_SetString(DokiError, "[PTRACE] Failed to allocate result matrix");
		return NULL;
	}
	m->elem = (int)id;
	Py_INCREF(cap);
	m->a = cap;
	return wrap_fmat(m);
}

static PyObject *doki_funmatrix_trace(PyObject *self, PyObject *args)
{
	PyObject *cap;
	int verbose;
	if (!PyArg_ParseTuple(args, "Op", &cap, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: funmatrix_trace(funmatrix, verbose)");
		return NULL;
	}
	fmat *m = get_fmat_msg(cap, "NULL pointer to matrix");
	if (!m)
		return NULL;
	const uint64_t mn = m->r <= m->c ? m->r : m->c;
	double complex acc = 0.0;
	for (uint64_t i = 0; i < mn; i++) {
		double complex v;
		int rc = fmat_get(m, i, i, &v);
		if (rc)
			return get_error(rc, "TRACE");
		if (isnan(creal(v)) || isnan(cimag(v))) {
			PyErr_SetString(DokiError, "[TRACE] Unexpected NAN value");
			return NULL;
		}
		acc += v;
	}
	return PyComplex_FromDoubles(creal(acc), cimag(acc));
}

/* Bytes held by a node and the nodes it references (funmatrix.c:1550-1567
 * counts operands recursively). */
static size_t fmat_mem(fmat *m, int depth)
{
	size_t s = sizeof(fmat);
	if (m->data)
		s += sizeof(fm_buf) + sizeof(double complex) * m->data->len;
	if (m->rho)
		s += sizeof(double complex) * m->r * m->r;
	s += sizeof(unsigned) * m->ntargets;
	if (depth < 256) {
		fmat *a = fmat_of(m->a), *b = fmat_of(m->b);
		if (a && m->kind != FM_DENSITY)
			s += fmat_mem(a, depth + 1);
		if (b)
			s += fmat_mem(b, depth + 1);
	}
	return s;
}

static PyObject *doki_funmatrix_mem(PyObject *self, PyObject *args)
{
	PyObject *cap;
	int verbose;
	if (!PyArg_ParseTuple(args, "Op", &cap, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: funmatrix_mem(fmatrix, verbose)");
		return NULL;
	}
	fmat *m = get_fmat_msg(cap, "NULL pointer to FMatrix");
	if (!m)
		return NULL;
	return PyLong_FromSize_t(fmat_mem(m, 0));
}

/* ---- lazy algebra (funmatrix.c:343-903, wrappers doki.c:1581-2055) ----- */

/* A op B node after the reference's operand checks; errors use its
 * "[TAG] ..." strings. */
static PyObject *fm_binary(PyObject *args, const char *syntax, const char *tag, int kind)
{
	PyObject *c1, *c2;
	int verbose;
	if (!PyArg_ParseTuple(args, "OOp", &c1, &c2, &verbose)) {
		PyErr_SetString(DokiError, syntax);
		return NULL;
	}
	fmat *a = (fmat *)PyCapsule_GetPointer(c1, CAP_FMAT);
	if (!a) {
		PyErr_Clear();
		PyErr_Format(DokiError, "[%s] The first operand is NULL", tag);
		return NULL;
	}
	fmat *b = (fmat *)PyCapsule_GetPointer(c2, CAP_FMAT);
	if (!b) {
		PyErr_Clear();
		PyErr_Format(DokiError, "[%s] The second operand is NULL", tag);
		return NULL;
	}
	uint64_t r, c;
	switch (kind) {
	case FM_ADD:
	case FM_SUB:
		if (a->r != b->r || a->c != b->c)
			goto misaligned;
		r = a->r;
		c = a->c;
		break;
	case FM_EWMUL:
		if (a->r == b->r && a->c == b->c) {
			r = a->r;
			c = a->c;
		} else if (a->r == 1 && b->c == 1) {
			/* row .* column is the outer product column * row */
			PyObject *t = c1;
			c1 = c2;
			c2 = t;
			kind = FM_MATMUL;
			r = b->r;
			c = a->c;
		} else if (b->r == 1 && a->c == 1) {
			kind = FM_MATMUL;
			r = a->r;
			c = b->c;
		} else {
			goto misaligned;
		}
		break;
	case FM_MATMUL:
		if (a->c != b->r)
			goto misaligned;
		r = a->r;
		c = b->c;
		break;
	default: /* FM_KRON */
		if ((a->r && b->r > UINT64_MAX / a->r) || (a->c && b->c > UINT64_MAX / a->c)) {
			PyErr_Format(DokiError, "[%s] Failed to allocate result matrix", tag);
			return NULL;
		}
		r = a->r * b->r;
		c = a->c * b->c;
		break;
	}
	fmat *m = fmat_new(kind, r, c);
	if (!m) {
		PyErr_Format(DokiError, "[%s] Failed to allocate result matrix", tag);
		return NULL;
	}
	Py_INCREF(c1);
	m->a = c1;
	Py_INCREF(c2);
	m->b = c2;
	return wrap_fmat(m);
misaligned:
	PyErr_Format(DokiError, "[%s] The operands are misalligned", tag);
	return NULL;
}

static PyObject *doki_funmatrix_add(PyObject *self, PyObject *args)
{
	return fm_binary(args, "Syntax: funmatrix_add(funmatrix1, funmatrix2, verbose)", "ADD",
			 FM_ADD);
}

static PyObject *doki_funmatrix_sub(PyObject *self, PyObject *args)
{
	return fm_binary(args, "Syntax: funmatrix_sub(funmatrix1, funmatrix2, verbose)", "SUB",
			 FM_SUB);
}

static PyObject *doki_funmatrix_matmul(PyObject *self, PyObject *args)
{
	return fm_binary(args, "Syntax: funmatrix_matmul(funmatrix1, funmatrix2, verbose)",
			 "MATMUL", FM_MATMUL);
}

static PyObject *doki_funmatrix_ewmul(PyObject *self, PyObject *args)
{
	return fm_binary(args, "Syntax: funmatrix_ewmul(funmatrix1, funmatrix2, verbose)",
			 "EWMUL", FM_EWMUL);
}

static PyObject *doki_funmatrix_kron(PyObject *self, PyObject *args)
{
	return fm_binary(args, "Syntax: funmatrix_kron(funmatrix1, funmatrix2, verbose)", "KRON",
			 FM_KRON);
}

/* Copy of a node with new modifiers: scalar product / division, transpose,
 * dagger.  The dagger flips both flags and leaves the scalar as it is, as
 * the reference's does. */
static PyObject *fm_modified(PyObject *cap, const char *tag, int op, double complex z)
{
	fmat *src = (fmat *)PyCapsule_GetPointer(cap, CAP_FMAT);
	if (!src) {
		PyErr_Clear();
		PyErr_Format(DokiError, op == 'T' || op == 'H' ? "[%s] The matrix is NULL" :
								   "[%s] The matrix operand is NULL",
			     tag);
		return NULL;
	}
	fmat *m = fmat_copy(src);
	if (!m) {
		PyErr_Format(DokiError, "[%s] Failed to allocate result matrix", tag);
		return NULL;
	}
	switch (op) {
	case '*':
		m->s = src->s * z;
		break;
	case '/':
		m->s = src->s / z;
		break;
	case 'T':
		m->transpose = !src->transpose;
		break;
	default: /* 'H' */
		m->transpose = !src->transpose;
		m->conjugate = !src->conjugate;
		break;
	}
	return wrap_fmat(m);
}

static int fm_scalar(PyObject *v, double complex *z)
{
	if (py_to_complex(v, z)) {
		PyErr_SetString(DokiError, "scalar is not a number");
		return -1;
	}
	return 0;
}

static PyObject *doki_funmatrix_scalar_mul(PyObject *self, PyObject *args)
{
	PyObject *cap, *raw;
	int verbose;
	double complex z;
	if (!PyArg_ParseTuple(args, "OOp", &cap, &raw, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: funmatrix_mul(funmatrix, scalar, verbose)");
		return NULL;
	}
	if (fm_scalar(raw, &z))
		return NULL;
	return fm_modified(cap, "SPROD", '*', z);
}

static PyObject *doki_funmatrix_scalar_div(PyObject *self, PyObject *args)
{
	PyObject *cap, *raw;
	int verbose;
	double complex z;
	if (!PyArg_ParseTuple(args, "OOp", &cap, &raw, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: funmatrix_div(funmatrix, scalar, verbose)");
		return NULL;
	}
	if (fm_scalar(raw, &z))
		return NULL;
	if (creal(z) == 0 && cimag(z) == 0) {
		PyErr_SetString(DokiError, "Dividing by zero");
		return NULL;
	}
	return fm_modified(cap, "SDIV", '/', z);
}

static PyObject *doki_funmatrix_transpose(PyObject *self, PyObject *args)
{
	PyObject *cap;
	int verbose;
	if (!PyArg_ParseTuple(args, "Op", &cap, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: funmatrix_transpose(funmatrix, verbose)");
		return NULL;
	}
	return fm_modified(cap, "TRANS", 'T', 0.0);
}

static PyObject *doki_funmatrix_dagger(PyObject *self, PyObject *args)
{
	PyObject *cap;
	int verbose;
	if (!PyArg_ParseTuple(args, "Op", &cap, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: funmatrix_dagger(funmatrix, verbose)");
		return NULL;
	}
	return fm_modified(cap, "HTRANS", 'H', 0.0);
}

static PyObject *doki_funmatrix_eyekron(PyObject *self, PyObject *args)
{
	PyObject *cap;
	unsigned int left, right;
	int verbose;
	if (!PyArg_ParseTuple(args, "OIIp", &cap, &left, &right, &verbose)) {
		PyErr_SetString(DokiError,
				"Syntax: funmatrix_eyekron(funmatrix, leftQubits, rightQubits, verbose)");
		return NULL;
	}
	fmat *u = get_fmat_msg(cap, "[EYEKRON] The matrix is NULL");
	if (!u)
		return NULL;
	const int lr = ilog2(u->r > u->c ? u->r : u->c);
	if ((uint64_t)left + right + (uint64_t)lr > 63) {
		PyErr_SetString(DokiError, "[EYEKRON] Failed to allocate result matrix");
		return NULL;
	}
	fmat *m = fmat_new(FM_EYEKRON, (1ull << left) * u->r * (1ull << right),
			   (1ull << left) * u->c * (1ull << right));
	if (!m) {
		PyErr_SetString(DokiError, "[EYEKRON] Failed to allocate result matrix");
		return NULL;
	}
	m->left = 1ull << left;
	m->right = 1ull << right;
	Py_INCREF(cap);
	m->a = cap;
	return wrap_fmat(m);
}

static PyObject *doki_funmatrix_projection(PyObject *self, PyObject *args)
{
	PyObject *cap;
	unsigned int qubit;
	int value, verbose;
	if (!PyArg_ParseTuple(args, "OIpp", &cap, &qubit, &value, &verbose)) {
		PyErr_SetString(DokiError,
				"Syntax: funmatrix_projection(funmatrix, qubit_id, value, verbose)");
		return NULL;
	}
	fmat *u = get_fmat_msg(cap, "[PROJ] The matrix is NULL");
	if (!u)
		return NULL;
	if (qubit > 63) {
		PyErr_SetString(DokiError, "[PROJ] Could not allocate data struct");
		return NULL;
	}
	fmat *m = fmat_new(FM_PROJECTION, u->r, u->c);
	if (!m) {
		PyErr_SetString(DokiError, "[PROJ] Failed to allocate result matrix");
		return NULL;
	}
	m->elem = (int)qubit;
	m->value = value ? 1 : 0;
	Py_INCREF(cap);
	m->a = cap;
	return wrap_fmat(m);
}

/* Qubit ids of a set for funmatrix_apply (doki.c:2331-2383); -1 on error. */
static int fm_apply_ids(PyObject *set, unsigned nq, const char *type_msg, const char *range_msg,
			uint64_t *mask)
{
	PyObject *it = PyObject_GetIter(set);
	if (!it)
		return -1;
	PyObject *v;
	while ((v = PyIter_Next(it))) {
		if (!PyLong_Check(v)) {
			Py_DECREF(v);
			Py_DECREF(it);
			PyErr_SetString(DokiError, type_msg);
			return -1;
		}
		const long q = PyLong_AsLong(v);
		Py_DECREF(v);
		if (q < 0 || (unsigned long)q >= nq) {
			Py_DECREF(it);
			PyErr_Clear();
			PyErr_SetString(DokiError, range_msg);
			return -1;
		}
		*mask |= 1ull << q;
	}
	Py_DECREF(it);
	return PyErr_Occurred() ? -1 : 0;
}

static PyObject *doki_funmatrix_apply(PyObject *self, PyObject *args)
{
	PyObject *scap, *gcap, *tlist, *cset, *aset;
	int verbose;
	if (!PyArg_ParseTuple(args, "OOOOOp", &scap, &gcap, &tlist, &cset, &aset, &verbose)) {
		PyErr_SetString(DokiError, "Syntax: funmatrix_apply(registry, gate, target_list, "
					   "control_set, anticontrol_set, verbose)");
		return NULL;
	}
	fmat *st = get_fmat_msg(scap, "NULL pointer to registry");
	if (!st)
		return NULL;
	fmat *g = get_fmat_msg(gcap, "NULL pointer to gate");
	if (!g)
		return NULL;
	if (st->c > 1) {
		PyErr_SetString(DokiError, "registry is not a column vector");
		return NULL;
	}
	if (g->c != g->r) {
		PyErr_SetString(DokiError, "gates have to be square matrices");
		return NULL;
	}
	if (g->r > st->r) {
		PyErr_SetString(DokiError, "gate is too big for this state vector");
		return NULL;
	}
	const int nq = ilog2(st->r);
	if (nq > 63 || st->r != (1ull << nq)) {
		PyErr_SetString(DokiError, "registry needs 2^n rows");
		return NULL;
	}
	const int ng = ilog2(g->r);
	if (ng > 63 || g->r != (1ull << ng)) {
		PyErr_SetString(DokiError, "gates need 2^n x 2^n elements");
		return NULL;
	}
	if (!PyList_Check(tlist)) {
		PyErr_SetString(DokiError, "target_list must be a list");
		return NULL;
	}
	const Py_ssize_t nt = PyList_Size(tlist);
	if (nt != ng) {
		PyErr_SetString(DokiError, "Wrong number of targets specified for that gate");
		return NULL;
	}
	const int have_c = PySet_Check(cset), have_a = PySet_Check(aset);
	if (!have_c && cset != Py_None) {
		PyErr_SetString(DokiError, "control_set must be a set or None");
		return NULL;
	}
	if (!have_a && aset != Py_None) {
		PyErr_SetString(DokiError, "anticontrol_set must be a set or None");
		return NULL;
	}
	uint64_t cmask = 0, amask = 0;
	if (have_c && PySet_Size(cset) > 0 &&
	    fm_apply_ids(cset, (unsigned)nq,
			 "control_set must be a set qubit ids (unsigned integers)",
			 "Control qubit out of range", &cmask))
		return NULL;
	if (have_a && PySet_Size(aset) > 0) {
		/* the reference tests each anticontrol for membership in the
		 * control argument, which fails unless that argument is a set */
		if (!have_c) {
			PyErr_SetString(DokiError, "A control cannot also be an anticontrol");
			return NULL;
		}
		PyObject *it = PyObject_GetIter(aset);
		if (!it)
			return NULL;
		PyObject *v;
		while ((v = PyIter_Next(it))) {
			if (!PyLong_Check(v)) {
				Py_DECREF(v);
				Py_DECREF(it);
				PyErr_SetString(DokiError, "anticontrol_set must be a set qubit ids "
							   "(unsigned integers)");
				return NULL;
			}
			const int clash = PySet_Contains(cset, v);
			const long q = PyLong_AsLong(v);
			Py_DECREF(v);
			if (clash) {
				Py_DECREF(it);
				PyErr_Clear();
				PyErr_SetString(DokiError, "A control cannot also be an anticontrol");
				return NULL;
			}
			if (q < 0 || (unsigned long)q >= (unsigned long)nq) {
				Py_DECREF(it);
				PyErr_Clear();
				PyErr_SetString(DokiError, "Anticontrol qubit out of range");
				return NULL;
			}
			amask |= 1ull << q;
		}
		Py_DECREF(it);
		if (PyErr_Occurred())
			return NULL;
	}
	unsigned *targets = (unsigned *)malloc(sizeof(unsigned) * (nt ? (size_t)nt : 1));
	if (!targets) {
		PyErr_SetString(DokiError, "Failed to allocate target array");
		return NULL;
	}
	for (Py_ssize_t k = 0; k < nt; k++) {
		PyObject *v = PyList_GetItem(tlist, k);
		if (!PyLong_Check(v)) {
			free(targets);
			PyErr_SetString(DokiError,
					"target_list must be a list of qubit ids (unsigned integers)");
			return NULL;
		}
		if ((have_c && PySet_Size(cset) > 0 && PySet_Contains(cset, v)) ||
		    (have_a && PySet_Size(aset) > 0 && PySet_Contains(aset, v))) {
			free(targets);
			PyErr_SetString(DokiError,
					"A target cannot also be a control or an anticontrol");
			return NULL;
		}
		const long q = PyLong_AsLong(v);
		if (q < 0 || q >= nq) {
			free(targets);
			PyErr_Clear();
			PyErr_SetString(DokiError, "Target qubit out of range");
			return NULL;
		}
		targets[k] = (unsigned)q;
	}
	fmat *m = fmat_new(FM_APPLY, st->r, 1);
	if (!m) {
		free(targets);
		PyErr_SetString(DokiError, "[FMAPPLY] Failed to allocate matrix");
		return NULL;
	}
	m->targets = targets;
	m->ntargets = (unsigned)nt;
	m->cmask = cmask;
	m->amask = amask;
	Py_INCREF(scap);
	m->a = scap;
	Py_INCREF(gcap);
	m->b = gcap;
	return wrap_fmat(m);
}

static PyMethodDef DokiMethods[] = {
	{ "gate_new", doki_gate_new, METH_VARARGS, "Create new gate" },
	{ "gate_get", doki_gate_get, METH_VARARGS, "Get matrix associated to gate" },
	{ "registry_new", doki_registry_new, METH_VARARGS, "Create new registry" },
	{ "registry_new_data", doki_registry_new_data, METH_VARARGS,
	  "Create new registry initialized with the specified values" },
	{ "registry_clone", doki_registry_clone, METH_VARARGS, "Clone a registry" },
	{ "registry_del", doki_registry_del, METH_VARARGS, "Destroy a registry" },
	{ "registry_get", doki_registry_get, METH_VARARGS, "Get value from registry" },
	{ "registry_apply", doki_registry_apply, METH_VARARGS, "Apply a gate" },
	{ "registry_join", doki_registry_join, METH_VARARGS, "Merges two registries" },
	{ "registry_measure", doki_registry_measure, METH_VARARGS,
	  "Measures and collapses specified qubits" },
	{ "registry_prob", doki_registry_prob, METH_VARARGS,
	  "Get the chances of obtaining 1 when measuring a certain qubit" },
	{ "registry_density", doki_registry_density, METH_VARARGS, "Get the density matrix" },
	{ "registry_mem", doki_registry_mem, METH_VARARGS,
	  "Get the memory allocated by this registry in bytes" },
	{ "funmatrix_create", doki_funmatrix_create, METH_VARARGS,
	  "Create a functional matrix from a matrix" },
	{ "funmatrix_identity", doki_funmatrix_identity, METH_VARARGS,
	  "Create an identity functional matrix of the specified number of qubits" },
	{ "funmatrix_statezero", doki_funmatrix_statezero, METH_VARARGS,
	  "State vector of n qubits at state zero" },
	{ "funmatrix_densityzero", doki_funmatrix_densityzero, METH_VARARGS,
	  "Density matrix of n qubits at state zero" },
	{ "funmatrix_hadamard", doki_funmatrix_hadamard, METH_VARARGS,
	  "Hadamard gate of the specified number of qubits" },
	{ "funmatrix_addcontrol", doki_funmatrix_addcontrol, METH_VARARGS,
	  "Same gate with a control qubit" },
	{ "funmatrix_get", doki_funmatrix_get, METH_VARARGS,
	  "Get a value from a functional matrix" },
	{ "funmatrix_add", doki_funmatrix_add, METH_VARARGS,
	  "Addition of two functional matrices" },
	{ "funmatrix_sub", doki_funmatrix_sub, METH_VARARGS,
	  "Subtraction of two functional matrices" },
	{ "funmatrix_scalar_mul", doki_funmatrix_scalar_mul, METH_VARARGS,
	  "Product of a scalar and a functional matrix" },
	{ "funmatrix_scalar_div", doki_funmatrix_scalar_div, METH_VARARGS,
	  "Division of a functional matrix by a scalar" },
	{ "funmatrix_matmul", doki_funmatrix_matmul, METH_VARARGS,
	  "Matrix product of two functional matrices" },
	{ "funmatrix_ewmul", doki_funmatrix_ewmul, METH_VARARGS,
	  "Element-wise product of two functional matrices" },
	{ "funmatrix_kron", doki_funmatrix_kron, METH_VARARGS,
	  "Kronecker product of two functional matrices" },
	{ "funmatrix_eyekron", doki_funmatrix_eyekron, METH_VARARGS,
	  "I(2^left) (x) U (x) I(2^right)" },
	{ "funmatrix_transpose", doki_funmatrix_transpose, METH_VARARGS,
	  "Transpose of a functional matrix" },
	{ "funmatrix_dagger", doki_funmatrix_dagger, METH_VARARGS,
	  "Conjugate transpose of a functional matrix" },
	{ "funmatrix_projection", doki_funmatrix_projection, METH_VARARGS,
	  "Projection of a functional matrix on one value of a qubit" },
	{ "funmatrix_shape", doki_funmatrix_shape, METH_VARARGS,
	  "Get a tuple with the shape of the matrix" },
	{ "funmatrix_partialtrace", doki_funmatrix_partialtrace, METH_VARARGS,
	  "Get the partial trace of a functional matrix" },
	{ "funmatrix_trace", doki_funmatrix_trace, METH_VARARGS,
	  "Get the trace of a functional matrix" },
	{ "funmatrix_apply", doki_funmatrix_apply, METH_VARARGS,
	  "Functional column vector after applying a gate to a functional state" },
	{ "funmatrix_mem", doki_funmatrix_mem, METH_VARARGS,
	  "Get the memory allocated by this FMatrix in bytes" },
	{ "registry_norm", doki_registry_norm, METH_VARARGS,
	  "(norm constant, 2-norm of the stored amplitudes) of a registry" },
	{ "registry_read_half", doki_registry_read_half, METH_VARARGS,
	  "Copy scale x the half of a registry at bit = value (distributed registers)" },
	{ "registry_replace_half", doki_registry_replace_half, METH_VARARGS,
	  "New registry with its half at bit = value replaced (distributed registers)" },
	{ "registry_apply_many", doki_registry_apply_many, METH_VARARGS,
	  "Queue every gate of a circuit given as flat arrays (serving form)" },
	{ "registry_get_all", doki_registry_get_all, METH_VARARGS,
	  "All amplitudes of a registry as a numpy array" },
	{ "registry_probs", doki_registry_probs, METH_VARARGS,
	  "P(qubit = 1) for every qubit" },
	{ "registry_precision", doki_registry_precision, METH_VARARGS,
	  "Storage precision of a registry (1 = complex64, 2 = complex128)" },
	{ "funmatrix_numpy", doki_funmatrix_numpy, METH_VARARGS,
	  "Materialise a functional matrix as a numpy array" },
	{ "engine_sync", doki_engine_sync, METH_VARARGS, "Wait for queued device work" },
	{ "engine_set_fusion", doki_engine_set_fusion, METH_VARARGS,
	  "Enable (default) or disable multi-gate sweep fusion" },
	{ "engine_stats", doki_engine_stats, METH_VARARGS,
	  "Kernel launches, sweeps, gates, host<->device bytes, tensor-core work and "
	  "tcgen05 sweep counts so far" },
	{ "registry_compare", doki_registry_compare, METH_VARARGS,
	  "(fidelity, max amplitude error) between two registries of equal size" },
	{ "engine_new_slot", doki_engine_new_slot, METH_VARARGS,
	  "Create a stream slot (own CUDA stream and scratch); returns its id" },
	{ "engine_set_slot", doki_engine_set_slot, METH_VARARGS,
	  "Select the slot new registries of this thread are created on" },
	{ "engine_get_slot", doki_engine_get_slot, METH_VARARGS,
	  "Slot new registries of this thread are created on" },
	{ "engine_stream", doki_engine_stream, METH_VARARGS,
	  "Address of the CUDA stream the engine queues its work on" },
	{ "registry_flush", doki_registry_flush, METH_VARARGS,
	  "Execute the gates queued on a registry now" },
	{ NULL, NULL, 0, NULL }
};

static struct PyModuleDef dokimodule = { PyModuleDef_HEAD_INIT, "doki", NULL, -1,
					 DokiMethods };

PyMODINIT_FUNC PyInit_doki(void)
{
	np_mod = PyImport_ImportModule("numpy");
	if (!np_mod)
		return NULL;
	np_ndarray = PyObject_GetAttrString(np_mod, "ndarray");
	np_complex128 = PyObject_GetAttrString(np_mod, "complex128");
	if (!np_ndarray || !np_complex128)
		return NULL;
	PyObject *m = PyModule_Create(&dokimodule);
	if (!m)
		return NULL;
	DokiError = PyErr_NewException("qsimov.doki.error", NULL, NULL);
	Py_XINCREF(DokiError);
	if (PyModule_AddObject(m, "error", DokiError) < 0) {
		Py_XDECREF(DokiError);
		Py_CLEAR(DokiError);
		Py_DECREF(m);
		return NULL;
	}
	return m;
}
