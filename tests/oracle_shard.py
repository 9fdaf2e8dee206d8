"""A doki-shaped module over the CPU oracle with the extra registry calls a
distributed register's shard makes (registry_apply_many, registry_norm,
registry_read_half, registry_replace_half, funmatrix_numpy) -- TEST
INFRASTRUCTURE: it lets the host logic of doki_b200.dist (EngineShard and
DistRegister) run on gloo ranks without a GPU, checked against the
single-register oracle."""
from __future__ import annotations

import ctypes

import numpy as np

from oracle import oracle as O


class OracleShardDoki(O.OracleDoki):
    """complex128 registers on the host; pointers are host addresses."""

    def registry_new(self, n, verbose=False, precision=2):
        assert precision == 2
        return super().registry_new(n, verbose)

    def registry_apply_many(self, reg, op_k, op_targets, op_controls, op_anticontrols,
                            op_matrix, matrices):
        for i in range(len(op_k)):
            k = int(op_k[i])
            m0 = int(op_matrix[i])
            g = self.gate_new(k, matrices[m0:m0 + (1 << (2 * k))]
                              .reshape(1 << k, 1 << k).tolist())
            cm, am = int(op_controls[i]), int(op_anticontrols[i])
            ctl = {q for q in range(reg.n) if (cm >> q) & 1}
            act = {q for q in range(reg.n) if (am >> q) & 1}
            # the engine applies gates to the stored amplitudes (a -> G a,
            # norm |G a|); the oracle applies them to a / norm, so hand it
            # the stored amplitudes with norm 1
            reg = self.registry_apply(O.OState(reg.n, reg.amp, 1.0), g,
                                      [int(t) for t in op_targets[i, :k]],
                                      ctl or None, act or None)
        return reg

    def registry_norm(self, reg):
        return reg.norm, float(np.linalg.norm(reg.amp))

    @staticmethod
    def _half_index(n, bit, value):
        j = np.arange(1 << (n - 1), dtype=np.int64)
        low = (1 << bit) - 1
        return ((j & ~low) << 1) | (value << bit) | (j & low)

    def registry_read_half(self, reg, bit, value, scale, ptr, on_device):
        assert not on_device
        half = np.ascontiguousarray(reg.vector()[self._half_index(reg.n, bit, value)] * scale)
        ctypes.memmove(ptr, half.ctypes.data, half.nbytes)

    def registry_replace_half(self, reg, bit, value, scale, ptr, on_device):
        assert not on_device
        cnt = 1 << (reg.n - 1)
        src = np.ctypeslib.as_array((ctypes.c_double * (2 * cnt)).from_address(ptr))
        out = reg.vector() * scale
        out[self._half_index(reg.n, bit, value)] = src.view(np.complex128)
        return O.OState(reg.n, np.ascontiguousarray(out), 1.0)

    def registry_probs(self, reg):
        # marginals relative to the stored norm, as the engine returns them
        p = np.abs(reg.amp / reg.norm) ** 2
        idx = np.arange(p.size)
        return [float(p[(idx >> q) & 1 == 1].sum()) for q in range(reg.n)]

    def funmatrix_numpy(self, fm):
        keep = O.kept_mask_after_traces(fm.state.n, fm.elems)
        return O.reduced_density(fm.state, keep)
