/*
 * doki -- CPython extension with the reference module's API (Mowstyl/Doki
 * src/doki/doki.c), backed by the B200 engine's C ABI (include/dokigpu.h).
 *
 * Same function names, positional argument formats, capsule names
 * ("qsimov.doki.state_vector", "qsimov.doki.gate", "qsimov.doki.funmatrix"),
 * exception object (qsimov.doki.error) and error strings as the reference
 * binding.  Differences, all strictly safer: out-of-range ids (registry_get,
 * registry_prob, funmatrix_partialtrace) and repeated targets raise instead
 * of reading out of bounds, and a registry passed to registry_del raises on
 * later use instead of being a dangling pointer.
 *
 * Extensions (optional trailing arguments never break positional calls):
 *   registry_new(n, verbose[, precision]) / registry_new_data(n, values,
 *   verbose[, precision]) -- precision 2 = complex128 (default), 1 = complex64;
 *   registry_get_all(reg, canonical) -> numpy complex128 array;
 *   registry_probs(reg) -> list of all P(q = 1);
 *   funmatrix_numpy(fm) -> numpy array of a density / reduced density matrix;
 *   registry_precision(reg); registry_flush(reg); registry_compare(a, b);
 *   engine_sync();
 *   engine_set_fusion(bool); engine_stats(); engine_stream();
 *   engine_new_slot(); engine_set_slot(slot); engine_get_slot().
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

enum {
	FM_CUSTOM = 1,
	FM_IDENTITY,
	FM_STATEZERO,
	FM_DENSITYZERO,
	FM_WALSH,
	FM_CU,
	FM_DENSITY,
	FM_PTRACE,
};

typedef struct fmat {
	int kind;
	uint64_t r, c;
	PyObject *parent; /* state capsule (DENSITY) / funmatrix capsule (CU, PTRACE) */
	int elem; /* PTRACE: qubit traced out of the parent */
	int hadamard;
	double complex *data; /* CUSTOM, row-major r x c */
	/* PTRACE chains rooted at a register: materialised reduced density */
	int mat_ready;
	uint64_t keep_mask;
	double complex *rho;
} fmat;

static void fmat_destroy(PyObject *cap)
{
	fmat *m = (fmat *)PyCapsule_GetPointer(cap, CAP_FMAT);
	if (!m) {
		PyErr_Clear();
		return;
	}
	Py_XDECREF(m->parent);
	free(m->data);
	free(m->rho);
	free(m);
}

static PyObject *wrap_fmat(fmat *m)
{
	PyObject *c = PyCapsule_New(m, CAP_FMAT, fmat_destroy);
	if (!c) {
		Py_XDECREF(m->parent);
		free(m->data);
		free(m);
	}
	return c;
}

static fmat *fmat_new(int kind, uint64_t r, uint64_t c)
{
	fmat *m = (fmat *)calloc(1, sizeof(fmat));
	if (m) {
		m->kind = kind;
		m->r = r;
		m->c = c;
	}
	return m;
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
	while ((1ull << l) < x)
		l++;
	return l;
}

/* If the chain of partial traces ends at a register's density matrix,
 * return its state capsule and the surviving-qubit mask. */
static PyObject *ptrace_root(fmat *m, uint64_t *keep)
{
	int elems[64], ne = 0;
	fmat *cur = m;
	while (cur->kind == FM_PTRACE && ne < 64) {
		elems[ne++] = cur->elem;
		cur = (fmat *)PyCapsule_GetPointer(cur->parent, CAP_FMAT);
		if (!cur) {
			PyErr_Clear();
			return NULL;
		}
	}
	if (cur->kind != FM_DENSITY)
		return NULL;
	dk_state *s = (dk_state *)PyCapsule_GetPointer(cur->parent, CAP_STATE);
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
	return cur->parent;
}

/* Element (i, j); returns 0 or a DK status (Python error not set). */
static int fmat_get(fmat *m, uint64_t i, uint64_t j, double complex *out)
{
	switch (m->kind) {
	case FM_CUSTOM:
		*out = m->data[i * m->c + j];
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
		fmat *u = (fmat *)PyCapsule_GetPointer(m->parent, CAP_FMAT);
		if (!u) {
			PyErr_Clear();
			return DK_ERR_ARG;
		}
		if (i < u->r || j < u->c) {
			*out = (i == j) ? 1.0 : 0.0;
			return 0;
		}
		return fmat_get(u, i - u->r, j - u->c, out);
	}
	case FM_DENSITY: {
		/* qops.c:266-293: psi_i conj(psi_j) */
		dk_state *s = (dk_state *)PyCapsule_GetPointer(m->parent, CAP_STATE);
		if (!s) {
			PyErr_Clear();
			return DK_ERR_ARG;
		}
		double ar, ai, br, bi;
		int rc = dk_get_amplitude(s, i, &ar, &ai);
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
				int rc = dk_reduced_density(s, keep, (double *)rho);
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
			int rc = dk_reduced_density_elem(s, keep, i, j, &re, &im);
			if (rc)
				return rc;
			*out = re + I * im;
			return 0;
		}
		/* generic lazy partial trace (funmatrix.c:920-944) */
		fmat *p = (fmat *)PyCapsule_GetPointer(m->parent, CAP_FMAT);
		if (!p) {
			PyErr_Clear();
			return DK_ERR_ARG;
		}
		double complex a, b;
		int rc = fmat_get(p, ins_bit(i, m->elem, 0), ins_bit(j, m->elem, 0), &a);
		if (rc)
			return rc;
		rc = fmat_get(p, ins_bit(i, m->elem, 1), ins_bit(j, m->elem, 1), &b);
		if (rc)
			return rc;
		*out = a + b;
		return 0;
	}
	default:
		return DK_ERR_ARG;
	}
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
	m->parent = cap;
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
	uint64_t l = 0, s = 0, g = 0, hi = 0, ho = 0;
	dk_get_stats(&l, &s, &g);
	dk_get_io_stats(&hi, &ho);
	return Py_BuildValue("{s:K,s:K,s:K,s:K,s:K}", "kernel_launches",
			     (unsigned long long)l, "sweeps", (unsigned long long)s, "gates",
			     (unsigned long long)g, "h2d_bytes", (unsigned long long)hi,
			     "d2h_bytes", (unsigned long long)ho);
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
	double complex *d = (double complex *)malloc(sizeof(double complex) * nr * nc);
	if (!m || !d) {
		free(m);
		free(d);
		PyErr_SetString(DokiError, "failed to allocate 2D matrix");
		return NULL;
	}
	for (Py_ssize_t i = 0; i < nr; i++) {
		row = PyList_GetItem(list, i);
		if (!PyList_Check(row) || PyList_Size(row) != nc) {
			free(m);
			free(d);
			PyErr_SetString(DokiError, "rows must be lists of the same size");
			return NULL;
		}
		for (Py_ssize_t j = 0; j < nc; j++)
			if (py_to_complex(PyList_GetItem(row, j), &d[i * nc + j])) {
				free(m);
				free(d);
				PyErr_SetString(DokiError, "matrix elements must be complex numbers");
				return NULL;
			}
	}
	m->data = d;
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
	fmat *u = (fmat *)PyCapsule_GetPointer(cap, CAP_FMAT);
	if (!u) {
		PyErr_SetString(DokiError, "NULL pointer to matrix");
		return NULL;
	}
	fmat *m = fmat_new(FM_CU, u->r * 2, u->c * 2);
	if (!m) {
		PyErr_SetString(DokiError, "NULL pointer to matrix");
		return NULL;
	}
	Py_INCREF(cap);
	m->parent = cap;
	return wrap_fmat(m);
}

static PyObject *get_error(int rc, const char *prefix)
{
	if (rc == DK_ERR_ARG)
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
	fmat *m = get_fmat(cap);
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
	if (m->r * m->c > (1ull << 28)) {
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
	if (m->kind == FM_PTRACE && m->mat_ready)
		memcpy(out, m->rho, sizeof(double complex) * m->r * m->c);
	else if (m->kind == FM_CUSTOM)
		memcpy(out, m->data, sizeof(double complex) * m->r * m->c);
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
	fmat *m = get_fmat(cap);
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
	fmat *p = (fmat *)PyCapsule_GetPointer(cap, CAP_FMAT);
	if (!p) {
		PyErr_SetString(DokiError, "[PTRACE] The matrix is NULL");
		return NULL;
	}
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
	m->parent = cap;
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
	fmat *m = get_fmat(cap);
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

static size_t fmat_mem(fmat *m)
{
	size_t s = sizeof(fmat);
	if (m->data)
		s += sizeof(double complex) * m->r * m->c;
	if (m->rho)
		s += sizeof(double complex) * m->r * m->r;
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
	fmat *m = (fmat *)PyCapsule_GetPointer(cap, CAP_FMAT);
	if (!m) {
		PyErr_SetString(DokiError, "NULL pointer to FMatrix");
		return NULL;
	}
	return PyLong_FromSize_t(fmat_mem(m));
}

/* Lazy FMatrix algebra (reference funmatrix.c:343-903) and funmatrix_apply
 * (qops.c:449-563) are outside this engine's scope. */
#define UNSUPPORTED(name)                                                          \
	static PyObject *doki_##name(PyObject *self, PyObject *args)               \
	{                                                                          \
		PyErr_SetString(DokiError, #name " is not supported by this engine"); \
		return NULL;                                                       \
	}
UNSUPPORTED(funmatrix_add)
UNSUPPORTED(funmatrix_sub)
UNSUPPORTED(funmatrix_scalar_mul)
UNSUPPORTED(funmatrix_scalar_div)
UNSUPPORTED(funmatrix_matmul)
UNSUPPORTED(funmatrix_ewmul)
UNSUPPORTED(funmatrix_kron)
UNSUPPORTED(funmatrix_eyekron)
UNSUPPORTED(funmatrix_transpose)
UNSUPPORTED(funmatrix_dagger)
UNSUPPORTED(funmatrix_projection)
UNSUPPORTED(funmatrix_apply)

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
	{ "funmatrix_add", doki_funmatrix_add, METH_VARARGS, "Not supported" },
	{ "funmatrix_sub", doki_funmatrix_sub, METH_VARARGS, "Not supported" },
	{ "funmatrix_scalar_mul", doki_funmatrix_scalar_mul, METH_VARARGS, "Not supported" },
	{ "funmatrix_scalar_div", doki_funmatrix_scalar_div, METH_VARARGS, "Not supported" },
	{ "funmatrix_matmul", doki_funmatrix_matmul, METH_VARARGS, "Not supported" },
	{ "funmatrix_ewmul", doki_funmatrix_ewmul, METH_VARARGS, "Not supported" },
	{ "funmatrix_kron", doki_funmatrix_kron, METH_VARARGS, "Not supported" },
	{ "funmatrix_eyekron", doki_funmatrix_eyekron, METH_VARARGS, "Not supported" },
	{ "funmatrix_transpose", doki_funmatrix_transpose, METH_VARARGS, "Not supported" },
	{ "funmatrix_dagger", doki_funmatrix_dagger, METH_VARARGS, "Not supported" },
	{ "funmatrix_projection", doki_funmatrix_projection, METH_VARARGS, "Not supported" },
	{ "funmatrix_shape", doki_funmatrix_shape, METH_VARARGS,
	  "Get a tuple with the shape of the matrix" },
	{ "funmatrix_partialtrace", doki_funmatrix_partialtrace, METH_VARARGS,
	  "Get the partial trace of a functional matrix" },
	{ "funmatrix_trace", doki_funmatrix_trace, METH_VARARGS,
	  "Get the trace of a functional matrix" },
	{ "funmatrix_apply", doki_funmatrix_apply, METH_VARARGS, "Not supported" },
	{ "funmatrix_mem", doki_funmatrix_mem, METH_VARARGS,
	  "Get the memory allocated by this FMatrix in bytes" },
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
	  "Kernel launches, sweeps, gates and host<->device bytes so far" },
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
