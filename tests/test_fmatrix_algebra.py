"""Lazy functional-matrix algebra against the reference module, on the host.

Both modules evaluate elements with C11 complex arithmetic in the same order
(reference funmatrix.c:238-340 getitem, qops.c:498-563 apply), so values are
compared bit for bit and errors by exception type and message.

Custom matrices given to the reference are square or single rows: it stores
``funmatrix_create`` data at ``[i * rows + j]`` (doki.c:1366), which overlaps
or overruns its buffer for any other shape.  Column vectors come from
``funmatrix_statezero`` and products with it.
"""
from __future__ import annotations

import numpy as np
import pytest


def _err(f):
    try:
        f()
    except Exception as e:  # noqa: BLE001
        return type(e).__module__ + "." + type(e).__name__, str(e)
    return None


def _mat(rng, r, c):
    m = rng.standard_normal((r, c)) + 1j * rng.standard_normal((r, c))
    return [[complex(x) for x in row] for row in m]


def _values(mod, fm):
    r, c = mod.funmatrix_shape(fm, False)
    return np.array([[mod.funmatrix_get(fm, i, j, False) for j in range(c)] for i in range(r)])


class Pair(tuple):
    """The same object built in the engine module (0) and the reference (1)."""


def both(dk, ref, name, *args):
    res = []
    for k, mod in enumerate((dk, ref)):
        conv = [a[k] if isinstance(a, Pair) else a for a in args]
        res.append(getattr(mod, name)(*conv))
    return Pair(res)


def same(dk, ref, p):
    va, vb = _values(dk, p[0]), _values(ref, p[1])
    assert va.shape == vb.shape
    assert np.array_equal(va.view(np.float64), vb.view(np.float64)), np.abs(va - vb).max()
    assert dk.funmatrix_trace(p[0], False) == ref.funmatrix_trace(p[1], False)


@pytest.fixture()
def rng():
    return np.random.default_rng(1234)


def test_binary_ops_match_reference(dk, ref, rng):
    A = both(dk, ref, "funmatrix_create", _mat(rng, 4, 4), False)
    B = both(dk, ref, "funmatrix_create", _mat(rng, 4, 4), False)
    for op in ("funmatrix_add", "funmatrix_sub", "funmatrix_matmul", "funmatrix_ewmul",
               "funmatrix_kron"):
        same(dk, ref, both(dk, ref, op, A, B, False))


def test_scalar_transpose_dagger_match_reference(dk, ref, rng):
    A = both(dk, ref, "funmatrix_create", _mat(rng, 4, 4), False)
    B = both(dk, ref, "funmatrix_create", _mat(rng, 4, 4), False)
    z = complex(0.3, -1.7)
    s = both(dk, ref, "funmatrix_scalar_mul", A, z, False)
    same(dk, ref, s)
    same(dk, ref, both(dk, ref, "funmatrix_scalar_div", A, z, False))
    same(dk, ref, both(dk, ref, "funmatrix_scalar_mul", A, 3, False))
    same(dk, ref, both(dk, ref, "funmatrix_scalar_div", A, 2.5, False))
    same(dk, ref, both(dk, ref, "funmatrix_transpose", A, False))
    same(dk, ref, both(dk, ref, "funmatrix_dagger", A, False))
    # the dagger keeps the node's scalar unconjugated, as the reference's does
    d = both(dk, ref, "funmatrix_dagger", s, False)
    same(dk, ref, d)
    a = np.array(_values(dk, A[0]))
    assert np.allclose(_values(dk, d[0]), z * a.conj().T)
    # modifiers on operation nodes and nested chains
    m = both(dk, ref, "funmatrix_matmul", A, B, False)
    same(dk, ref, both(dk, ref, "funmatrix_transpose", m, False))
    t = both(dk, ref, "funmatrix_dagger", both(dk, ref, "funmatrix_scalar_mul", m, 1j, False),
             False)
    same(dk, ref, both(dk, ref, "funmatrix_transpose", t, False))
    same(dk, ref, both(dk, ref, "funmatrix_add", t, both(dk, ref, "funmatrix_transpose", B,
                                                          False), False))


def test_nonsquare_shapes_match_reference(dk, ref, rng):
    row = both(dk, ref, "funmatrix_create", _mat(rng, 1, 4), False)
    col = both(dk, ref, "funmatrix_statezero", 2, False)
    H = both(dk, ref, "funmatrix_hadamard", 2, False)
    v = both(dk, ref, "funmatrix_matmul", H, col, False)       # 4 x 1
    same(dk, ref, v)
    same(dk, ref, both(dk, ref, "funmatrix_ewmul", row, v, False))  # row .* column
    same(dk, ref, both(dk, ref, "funmatrix_ewmul", v, row, False))  # column .* row
    same(dk, ref, both(dk, ref, "funmatrix_kron", v, row, False))   # 4 x 4 outer
    same(dk, ref, both(dk, ref, "funmatrix_kron", row, H, False))   # 4 x 16
    same(dk, ref, both(dk, ref, "funmatrix_matmul", row, H, False))  # 1 x 4


def test_eyekron_matches_reference(dk, ref, rng):
    U = both(dk, ref, "funmatrix_create", _mat(rng, 2, 2), False)
    for left, right in ((0, 0), (1, 0), (0, 2), (2, 1)):
        same(dk, ref, both(dk, ref, "funmatrix_eyekron", U, left, right, False))
    V = both(dk, ref, "funmatrix_dagger", both(dk, ref, "funmatrix_create", _mat(rng, 4, 4),
                                                 False), False)
    same(dk, ref, both(dk, ref, "funmatrix_eyekron", V, 1, 1, False))


# funmatrix_projection and funmatrix_apply are not called on the reference:
# its wrappers parse "p" arguments into 1-byte bools (doki.c:2021, 2226), and
# the int stores overwrite neighbouring locals (qubit_id, the state capsule),
# so on this build they mask the wrong qubit, reject valid capsules or crash.
# They are checked against restatements of their element rules instead.

def _projection_rule(a, q, v):
    """funmatrix.c:862-890: rows whose bit q differs from v are zero."""
    out = a.copy()
    out[[((i >> q) & 1) != v for i in range(a.shape[0])], :] = 0
    return out


def _apply_rule(x, g, targets, controls, anticontrols):
    """qops.c:498-563, element by element in the reference's order."""
    cm = sum(1 << c for c in (controls or ()))
    am = sum(1 << c for c in (anticontrols or ()))
    out = []
    for i in range(len(x)):
        if (i & cm) != cm or (i & am):
            out.append(x[i])
            continue
        row = sum(((i >> t) & 1) << k for k, t in enumerate(targets))
        acc, reg = 0j, i
        for n in range(g.shape[0]):
            for k, t in enumerate(targets):
                reg = reg | (1 << t) if (n >> k) & 1 else reg & ~(1 << t)
            acc = acc + x[reg] * g[row, n]
        out.append(acc)
    return np.array(out)


def test_projection_rule(dk, rng):
    m = _mat(rng, 8, 8)
    M = dk.funmatrix_create(m, False)
    a = np.array(m)
    for q in range(3):
        for v in (False, True):
            got = _values(dk, dk.funmatrix_projection(M, q, v, False))
            assert np.array_equal(got, _projection_rule(a, q, v))
    T = dk.funmatrix_projection(dk.funmatrix_dagger(M, False), 2, True, False)
    assert np.array_equal(_values(dk, T), _projection_rule(a.conj().T, 2, True))
    S = dk.funmatrix_scalar_mul(T, -2j, False)
    assert np.array_equal(_values(dk, S), _projection_rule(a.conj().T, 2, True) * -2j)


def test_apply_rule(dk, ref, rng):
    n = 4
    m = _mat(rng, 1 << n, 1 << n)
    M = dk.funmatrix_create(m, False)
    psi = dk.funmatrix_matmul(M, dk.funmatrix_statezero(n, False), False)
    x = _values(dk, psi)[:, 0]
    # the state vector itself is checked against the reference's matmul
    R = ref.funmatrix_matmul(ref.funmatrix_create(m, False), ref.funmatrix_statezero(n, False),
                             False)
    assert np.array_equal(x, _values(ref, R)[:, 0])
    g1, g2 = _mat(rng, 2, 2), _mat(rng, 4, 4)
    G1, G2 = dk.funmatrix_create(g1, False), dk.funmatrix_create(g2, False)
    H = dk.funmatrix_hadamard(1, False)
    h = _values(dk, H)
    cases = [
        (G1, g1, [0], None, None),
        (G1, g1, [3], {1}, None),
        (G1, g1, [2], {0, 3}, set()),
        (G1, g1, [1], set(), {2}),
        (G1, g1, [0], {3}, {1, 2}),
        (G2, g2, [0, 2], None, None),
        (G2, g2, [3, 1], {0}, {2}),
        (H, h, [2], None, None),
    ]
    cur, want_cur = psi, x
    for G, g, t, c, a in cases:
        g = np.array(g)
        r = dk.funmatrix_apply(psi, G, t, c, a, False)
        assert dk.funmatrix_shape(r, False) == (1 << n, 1)
        assert np.array_equal(_values(dk, r)[:, 0], _apply_rule(x, g, t, c, a))
        cur = dk.funmatrix_apply(cur, G, t, c, a, False)
        want_cur = _apply_rule(want_cur, g, t, c, a)
    assert np.allclose(_values(dk, cur)[:, 0], want_cur, rtol=0, atol=1e-12)
    # a unitary on a normalised state keeps the norm
    u = dk.funmatrix_apply(dk.funmatrix_statezero(3, False), dk.funmatrix_hadamard(2, False),
                           [0, 2], None, None, False)
    assert np.isclose(np.vdot(_values(dk, u)[:, 0], _values(dk, u)[:, 0]).real, 1.0)


def test_bulk_export_applies_modifiers(dk, rng):
    m = _mat(rng, 4, 4)
    A = dk.funmatrix_create(m, False)
    a = np.array(m)
    assert np.array_equal(dk.funmatrix_numpy(A), a)
    assert np.array_equal(dk.funmatrix_numpy(dk.funmatrix_dagger(A, False)), a.conj().T)
    assert np.array_equal(dk.funmatrix_numpy(dk.funmatrix_scalar_mul(A, 2, False)), 2 * a)
    B = dk.funmatrix_matmul(A, dk.funmatrix_transpose(A, False), False)
    assert np.allclose(dk.funmatrix_numpy(B), a @ a.T, atol=1e-13)


def _pairs_for_errors(dk, ref, rng):
    sq = _mat(rng, 2, 2)
    return {
        "A2": both(dk, ref, "funmatrix_create", sq, False),
        "A4": both(dk, ref, "funmatrix_identity", 2, False),
        "row": both(dk, ref, "funmatrix_create", [[1, 2, 3, 4]], False),
        "col": both(dk, ref, "funmatrix_statezero", 2, False),
        "nan": both(dk, ref, "funmatrix_create", [[float("nan"), 1], [0, 1]], False),
        "gate": Pair([dk.gate_new(1, sq, False), ref.gate_new(1, sq, False)]),
    }


ERROR_CASES = [
    ("funmatrix_add", ("A2", "A4")),
    ("funmatrix_sub", ("A4", "A2")),
    ("funmatrix_matmul", ("A4", "A2")),
    ("funmatrix_ewmul", ("A2", "A4")),
    ("funmatrix_add", ("gate", "A2")),
    ("funmatrix_sub", ("A2", "gate")),
    ("funmatrix_matmul", ("gate", "A2")),
    ("funmatrix_ewmul", ("A2", "gate")),
    ("funmatrix_kron", ("gate", "A2")),
    ("funmatrix_kron", ("A2", "gate")),
    ("funmatrix_transpose", ("gate",)),
    ("funmatrix_dagger", ("gate",)),
    ("funmatrix_scalar_mul", ("gate", 2)),
    ("funmatrix_scalar_mul", ("A2", "x")),
    ("funmatrix_scalar_div", ("A2", 0)),
    ("funmatrix_scalar_div", ("A2", 0j)),
    ("funmatrix_scalar_div", ("gate", 1)),
    ("funmatrix_eyekron", ("gate", 1, 1)),
]

# Messages of the reference's funmatrix_apply / funmatrix_projection checks
# (doki.c:2016-2055, 2217-2437), in the order it makes them.
RULE_ERRORS = [
    ("funmatrix_projection", ("gate", 0, True), "[PROJ] The matrix is NULL"),
    ("funmatrix_apply", ("gate", "A2", [0], None, None), "NULL pointer to registry"),
    ("funmatrix_apply", ("col", "gate", [0], None, None), "NULL pointer to gate"),
    ("funmatrix_apply", ("A4", "A2", [0], None, None), "registry is not a column vector"),
    ("funmatrix_apply", ("col", "row", [0], None, None), "gates have to be square matrices"),
    ("funmatrix_apply", ("col2", "A4", [0, 1], None, None),
     "gate is too big for this state vector"),
    ("funmatrix_apply", ("col3", "A2", [0], None, None), "registry needs 2^n rows"),
    ("funmatrix_apply", ("col", "A3", [0], None, None), "gates need 2^n x 2^n elements"),
    ("funmatrix_apply", ("col", "A2", (0,), None, None), "target_list must be a list"),
    ("funmatrix_apply", ("col", "A2", [0, 1], None, None),
     "Wrong number of targets specified for that gate"),
    ("funmatrix_apply", ("col", "A2", [0], [1], None), "control_set must be a set or None"),
    ("funmatrix_apply", ("col", "A2", [0], None, [1]),
     "anticontrol_set must be a set or None"),
    ("funmatrix_apply", ("col", "A2", [0], None, {1}),
     "A control cannot also be an anticontrol"),
    ("funmatrix_apply", ("col", "A2", [0], {1}, {1}),
     "A control cannot also be an anticontrol"),
    ("funmatrix_apply", ("col", "A2", [0], {0}, None),
     "A target cannot also be a control or an anticontrol"),
    ("funmatrix_apply", ("col", "A2", [0], set(), {0}),
     "A target cannot also be a control or an anticontrol"),
    ("funmatrix_apply", ("col", "A2", [2], None, None), "Target qubit out of range"),
    ("funmatrix_apply", ("col", "A2", [0], {5}, None), "Control qubit out of range"),
    ("funmatrix_apply", ("col", "A2", [0], {1}, {7}), "Anticontrol qubit out of range"),
    ("funmatrix_apply", ("col", "A2", ["a"], None, None),
     "target_list must be a list of qubit ids (unsigned integers)"),
    ("funmatrix_apply", ("col", "A2", [0], {"a"}, None),
     "control_set must be a set qubit ids (unsigned integers)"),
    ("funmatrix_apply", ("col", "A2", [0], set(), {"a"}),
     "anticontrol_set must be a set qubit ids (unsigned integers)"),
]


@pytest.mark.parametrize("name,spec,msg", RULE_ERRORS)
def test_apply_projection_errors(dk, name, spec, msg):
    sq = [[1, 2], [3, 4]]
    objs = {
        "A2": dk.funmatrix_create(sq, False),
        "A3": dk.funmatrix_create([[1, 0, 0], [0, 1, 0], [0, 0, 1]], False),
        "A4": dk.funmatrix_identity(2, False),
        "row": dk.funmatrix_create([[1, 2, 3, 4]], False),
        "col": dk.funmatrix_statezero(2, False),
        "col2": dk.funmatrix_statezero(1, False),
        "col3": dk.funmatrix_create([[1], [2], [3]], False),
        "gate": dk.gate_new(1, sq, False),
    }
    args = [objs[s] if isinstance(s, str) and s in objs else s for s in spec]
    with pytest.raises(dk.error) as e:
        getattr(dk, name)(*args, False)
    assert str(e.value) == msg


@pytest.mark.parametrize("name,spec", ERROR_CASES)
def test_algebra_errors_match_reference(dk, ref, rng, name, spec):
    objs = _pairs_for_errors(dk, ref, rng)
    args = [objs[s] if isinstance(s, str) and s in objs else s for s in spec]
    got = []
    for k, mod in enumerate((dk, ref)):
        conv = [a[k] if isinstance(a, Pair) else a for a in args]
        got.append(_err(lambda: getattr(mod, name)(*conv, False)))
    assert got[0] is not None
    assert got[0] == got[1]


@pytest.mark.parametrize("expr", ["add", "matmul", "kron", "dagger_add"])
def test_element_errors_match_reference(dk, ref, rng, expr):
    objs = _pairs_for_errors(dk, ref, rng)
    nan, A2 = objs["nan"], objs["A2"]
    if expr == "add":
        p = both(dk, ref, "funmatrix_add", A2, nan, False)
    elif expr == "matmul":
        p = both(dk, ref, "funmatrix_matmul", nan, A2, False)
    elif expr == "kron":
        p = both(dk, ref, "funmatrix_kron", A2, nan, False)
    else:
        p = both(dk, ref, "funmatrix_dagger", both(dk, ref, "funmatrix_add", nan, A2, False),
                 False)
    for call in (lambda m, x: m.funmatrix_get(x, 0, 0, False),
                 lambda m, x: m.funmatrix_trace(x, False)):
        a = _err(lambda: call(dk, p[0]))
        b = _err(lambda: call(ref, p[1]))
        assert a is not None and a == b
    # the NaN leaf itself
    assert _err(lambda: dk.funmatrix_get(nan[0], 0, 0, False)) == \
        _err(lambda: ref.funmatrix_get(nan[1], 0, 0, False))


def test_nodes_release_their_operands(dk):
    """Every node holds references to its operands only while it lives."""
    import gc
    import sys
    A = dk.funmatrix_create([[1, 2], [3, 4]], False)
    B = dk.funmatrix_identity(1, False)
    col = dk.funmatrix_statezero(1, False)
    base = [sys.getrefcount(o) for o in (A, B, col)]
    for _ in range(50):
        x = dk.funmatrix_add(A, B, False)
        y = dk.funmatrix_dagger(x, False)
        z = dk.funmatrix_scalar_mul(y, 2j, False)
        k = dk.funmatrix_kron(z, A, False)
        e = dk.funmatrix_eyekron(A, 1, 1, False)
        p = dk.funmatrix_projection(k, 1, True, False)
        ap = dk.funmatrix_apply(col, A, [0], None, None, False)
        t = dk.funmatrix_partialtrace(k, 0, False)
        with pytest.raises(dk.error):
            dk.funmatrix_apply(col, A, [0], {5}, None, False)
        dk.funmatrix_get(p, 1, 1, False)
        dk.funmatrix_trace(t, False)
        dk.funmatrix_numpy(ap)
        del x, y, z, k, e, p, ap, t
    gc.collect()
    assert [sys.getrefcount(o) for o in (A, B, col)] == base
