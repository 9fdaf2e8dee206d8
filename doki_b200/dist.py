"""Distributed register: one n-qubit register sharded over 2^g ranks.

The reference keeps a register in one host allocation (its chunked
``vector**`` layout, qstate.h:44-59, is always one chunk in practice,
platform.h:255), so it stops at one machine's memory.  Here rank r holds the
amplitudes whose top g index bits equal r, as an ordinary engine register of
nl = n - g qubits on its own GPU; a register of 33 qubits complex128 and
beyond is spread over the GPUs of a node.

Layout.  Position p of the global index: positions 0 .. nl-1 are the bits
of a rank's local register, positions nl .. n-1 the bits of the rank
number.  ``perm[p]`` is the logical qubit (the reference's qubit id) held at
position p; it changes as rank qubits are swapped in.

Values.  A shard holds a local register whose normalised amplitudes v_r are
scaled by a host weight w_r >= 0: the amplitude at global index (r, j) is
w_r v_r[j], with sum_r w_r^2 = 1.  Gates on local positions run on the
local register; a gate's controls on rank positions are decided per rank
(a failed control leaves the rank's part untouched).  The reference
renormalises after every gate (qops.c:256-258); here each rank's weight
grows by |G v_r| and all weights are divided by their root sum of squares,
which gives the same normalised register for unitary and non-unitary
gates alike.

Exchange.  A gate whose target lies on a rank position first swaps that
position with a local one: rank r and its partner r ^ 2^b exchange the
half of their local amplitudes whose local bit p equals the complement of
their rank bit b (one send and one receive of 2^(nl-1) amplitudes each,
torch.distributed point-to-point: NCCL between GPUs of a node, gloo on CPU),
and each rebuilds its register from its kept half and the received half.
No collective touches the amplitudes; marginals, measurement and the
reduced density matrix all-reduce n doubles, a few scalars or one 4^k
matrix.

Measurement (reference doki.c:1097-1157, one qubit at a time, highest
first): P(q = 1) is all-reduced; every rank takes the same decision.  A
local qubit collapses every shard (its weight scaled by the shard's share of
the selected outcome); a qubit on a rank position zeroes the weight of the
ranks on the other side and freezes that rank bit.

The local register is any object with the shard interface of
:class:`EngineShard`; the product binds it to the engine (``doki`` module)
on the rank's GPU.
"""
from __future__ import annotations

import math
from typing import Dict, List, Optional, Sequence

import numpy as np


class EngineShard:
    """The local part of a distributed register: an engine register of nl
    qubits and the bookkeeping of its normalisation.

    The engine stores raw amplitudes a with a norm constant c (logical =
    a / c, reference qstate.h:84-86); the shard's normalised amplitudes are
    v = a / |a|.  `d` is the doki module (or any module with the same
    registry_* functions, including registry_norm, registry_read_half,
    registry_replace_half and registry_apply_many)."""

    def __init__(self, d, nl: int, precision: int = 2, device: bool = False, reg=None):
        self.d = d
        self.nl = nl
        self.precision = precision
        self.device = device
        self.reg = reg if reg is not None else d.registry_new(nl, False, precision)
        self._stored = self._norms()[1]

    @property
    def dtype(self):
        return np.complex128 if self.precision == 2 else np.complex64

    def _norms(self):
        return self.d.registry_norm(self.reg)

    def apply(self, flat_arrays) -> None:
        """Queue gates on local positions (the flat arrays of
        registry_apply_many)."""
        self.reg = self.d.registry_apply_many(self.reg, *flat_arrays)

    def growth(self) -> float:
        """|G v| of the gates queued since the last call (the stored
        amplitudes evolve as a -> G a, so the ratio of their norms)."""
        _, stored = self._norms()
        f = stored / self._stored if self._stored > 0 else 0.0
        self._stored = stored
        return f

    def probs(self) -> np.ndarray:
        """P(local position p = 1) of v for every p."""
        c, stored = self._norms()
        if stored == 0.0:
            return np.zeros(self.nl)
        return np.asarray(self.d.registry_probs(self.reg)) * (c / stored) ** 2

    def _buffer(self, count):
        if self.device:
            import torch
            return torch.empty(count, dtype=torch.complex128 if self.precision == 2
                               else torch.complex64, device="cuda")
        return np.empty(count, dtype=self.dtype)

    @staticmethod
    def _ptr(buf):
        return buf.data_ptr() if hasattr(buf, "data_ptr") else buf.ctypes.data

    def read_half(self, pos: int, value: int, scale: float):
        """scale x v over the local indices whose bit `pos` equals `value`."""
        c, stored = self._norms()
        buf = self._buffer(1 << (self.nl - 1))
        k = scale * c / stored if stored > 0 else 0.0
        self.d.registry_read_half(self.reg, pos, value, k, self._ptr(buf), self.device)
        return buf

    def replace_half(self, pos: int, value: int, scale: float, buf) -> float:
        """The local amplitudes become u = (`buf` where bit `pos` = `value`,
        scale x v elsewhere); returns |u| (v becomes u / |u|)."""
        c, stored = self._norms()
        k = scale * c / stored if stored > 0 else 0.0
        self.reg = self.d.registry_replace_half(self.reg, pos, value, k, self._ptr(buf),
                                                self.device)
        self._stored = self._norms()[1]
        return self._stored

    def collapse(self, pos: int, outcome: int) -> float:
        """Keep the half of v where local position `pos` equals `outcome`
        (the register loses that position); returns that half's share of
        |v|^2 (0: the rank's part vanishes, its content is then
        immaterial)."""
        p1 = float(self.probs()[pos])
        share = p1 if outcome else 1.0 - p1
        if self.nl == 1:
            self.reg = None
            self.nl = 0
            return share
        # the collapse itself picks the half; the roll forces the outcome
        # whenever that half holds amplitude
        roll = 0.0 if outcome else math.nextafter(1.0, 0.0)
        new, _ = self.d.registry_measure(self.reg, 1 << pos, [roll], -1, False)
        self.reg = new
        self.nl -= 1
        self._stored = self._norms()[1]
        return share

    def reduced_density(self, keep_positions: Sequence[int]) -> np.ndarray:
        """Reduced density matrix of v over the given local positions (index
        bits in increasing position order)."""
        rho = self.d.registry_density(self.reg, False)
        keep = set(keep_positions)
        for p in range(self.nl - 1, -1, -1):
            if p not in keep:
                rho = self.d.funmatrix_partialtrace(rho, p, False)
        m = np.asarray(self.d.funmatrix_numpy(rho))
        c, stored = self._norms()
        return m * (c / stored) ** 2 if stored > 0 else m * 0.0

    def amplitudes(self) -> np.ndarray:
        """v as a host array (small registers)."""
        c, stored = self._norms()
        a = np.asarray(self.d.registry_get_all(self.reg, False))
        return a * (c / stored) if stored > 0 else a * 0.0


def _flat_ops(ops, nl):
    """(matrix, local targets, local control mask, local anticontrol mask)
    list -> the flat arrays of registry_apply_many."""
    n = len(ops)
    k = np.zeros(n, dtype=np.uint32)
    tg = np.zeros((n, 3), dtype=np.uint32)
    cm = np.zeros(n, dtype=np.uint64)
    am = np.zeros(n, dtype=np.uint64)
    mi = np.zeros(n, dtype=np.uint64)
    mats, off = [], 0
    for i, (mat, targets, c, a) in enumerate(ops):
        k[i] = len(targets)
        tg[i, :len(targets)] = targets
        cm[i], am[i], mi[i] = c, a, off
        m = np.ascontiguousarray(mat, dtype=np.complex128).reshape(-1)
        mats.append(m)
        off += m.size
    matrices = np.concatenate(mats) if mats else np.zeros(1, dtype=np.complex128)
    return k, tg, cm, am, mi, matrices


class DistRegister:
    """An n-qubit register over the ranks of `group` (a power of two).

    `make_shard(nl)` returns this rank's local register of nl qubits in
    |0..0> (an :class:`EngineShard` in the product).  `comm` is
    torch.distributed (or an object with the same all_reduce /
    batch_isend_irecv / P2POp / isend / irecv / ReduceOp)."""

    def __init__(self, n: int, make_shard, comm, group=None):
        self.comm = comm
        self.group = group
        self.rank = comm.get_rank(group)
        self.world = comm.get_world_size(group)
        g = self.world.bit_length() - 1
        if 1 << g != self.world:
            raise ValueError("the number of ranks must be a power of two")
        if n <= g:
            raise ValueError("more rank bits than qubits")
        self.n = n
        self.nl = n - g
        self.shard = make_shard(self.nl)
        # |0..0>: the whole amplitude sits on rank 0
        self.w = 1.0 if self.rank == 0 else 0.0
        self.perm: List[int] = list(range(n))  # position -> logical qubit
        self.rank_bits: List[int] = list(range(g))  # rank bit of each rank position
        self.frozen: Dict[int, int] = {}  # measured rank bit -> its fixed value
        self.pending: List = []
        self.exchanges = 0
        # NCCL reduces device tensors; gloo host tensors
        self.cuda_collectives = comm.get_backend(group) == "nccl"

    # -- layout -----------------------------------------------------------
    def position(self, q: int) -> int:
        return self.perm.index(q)

    def _is_local(self, p: int) -> bool:
        return p < self.nl

    def _rank_bit(self, p: int) -> int:
        return self.rank_bits[p - self.nl]

    def _my_bit(self, p: int) -> int:
        return (self.rank >> self._rank_bit(p)) & 1

    # -- collectives --------------------------------------------------------
    def _allreduce(self, arr: np.ndarray) -> np.ndarray:
        import torch
        t = torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float64))
        if self.cuda_collectives:
            t = t.cuda()
        self.comm.all_reduce(t, op=self.comm.ReduceOp.SUM, group=self.group)
        return t.cpu().numpy()

    def _exchange(self, partner: int, send, recv) -> None:
        import torch
        s = send if hasattr(send, "data_ptr") else torch.from_numpy(send)
        r = recv if hasattr(recv, "data_ptr") else torch.from_numpy(recv)
        s, r = torch.view_as_real(s), torch.view_as_real(r)
        ops = [self.comm.P2POp(self.comm.isend, s, partner, self.group),
               self.comm.P2POp(self.comm.irecv, r, partner, self.group)]
        for req in self.comm.batch_isend_irecv(ops):
            req.wait()
        self.exchanges += 1

    # -- gates --------------------------------------------------------------
    def apply(self, gate: np.ndarray, targets: Sequence[int],
              controls: Optional[set] = None, anticontrols: Optional[set] = None) -> None:
        """registry_apply (qops.c:176-261) on the distributed register:
        `targets[0]` is the least significant bit of the gate index."""
        controls, anticontrols = set(controls or ()), set(anticontrols or ())
        for q in targets:
            p = self.position(q)
            if not self._is_local(p):
                self._swap_in(p, avoid=set(targets) | controls | anticontrols)
        lt = [self.position(q) for q in targets]
        cm = am = 0
        active = True
        for q in controls:
            p = self.position(q)
            if self._is_local(p):
                cm |= 1 << p
            elif self._my_bit(p) != 1:
                active = False
        for q in anticontrols:
            p = self.position(q)
            if self._is_local(p):
                am |= 1 << p
            elif self._my_bit(p) != 0:
                active = False
        if active and self.w > 0.0:
            self.pending.append((gate, lt, cm, am))

    def _flush(self) -> None:
        """Run the queued local gates and renormalise over all ranks."""
        if self.pending and self.w > 0.0:
            self.shard.apply(_flat_ops(self.pending, self.nl))
            self.w *= self.shard.growth()
        self.pending = []
        z = math.sqrt(float(self._allreduce(np.array([self.w * self.w]))[0]))
        if z == 0.0:
            raise ZeroDivisionError("the register's norm vanished")
        self.w /= z

    def _swap_in(self, pg: int, avoid: set) -> None:
        """Swap rank position pg with the highest local position whose qubit
        is not in `avoid` (exchange with the partner rank)."""
        self._flush()
        pl = max(p for p in range(self.nl) if self.perm[p] not in avoid)
        b = self._rank_bit(pg)
        y = (self.rank >> b) & 1
        partner = self.rank ^ (1 << b)
        send = self.shard.read_half(pl, 1 - y, self.w)
        recv = self.shard._buffer(1 << (self.nl - 1))
        self._exchange(partner, send, recv)
        self.w = self.shard.replace_half(pl, 1 - y, self.w, recv)
        self.perm[pl], self.perm[pg] = self.perm[pg], self.perm[pl]

    # -- reads --------------------------------------------------------------
    def probs(self) -> np.ndarray:
        """P(q = 1) for every logical qubit q (qops.c:72-95)."""
        self._flush()
        local = self.shard.probs() if self.w > 0 else np.zeros(self.nl)
        vec = np.zeros(self.n)
        for p in range(self.n):
            if self._is_local(p):
                vec[self.perm[p]] = self.w * self.w * local[p]
            else:
                vec[self.perm[p]] = self.w * self.w * self._my_bit(p)
        return self._allreduce(vec)

    def measure(self, mask: int, rolls: Sequence[float]) -> List[Optional[bool]]:
        """registry_measure (doki.c:1023-1192): qubits n-1 .. 0 set in `mask`,
        one roll each; entry i of the result is qubit n-1-i (None when not
        measured).  The register keeps the unmeasured qubits, renumbered as
        the reference's collapsed register."""
        n0 = self.n
        out: List[Optional[bool]] = [None] * n0
        rid = 0
        for i in range(n0):
            q = n0 - 1 - i
            if not (mask >> q) & 1:
                continue
            roll = float(rolls[rid])
            rid += 1
            if not 0.0 <= roll < 1.0:
                raise ValueError("roll not in interval [0, 1)!")
            p1 = float(self.probs()[q])
            bit = 1 if p1 > roll else 0
            out[i] = bool(bit)
            self._collapse(q, bit, p1 if bit else 1.0 - p1)
        return out

    def _collapse(self, q: int, bit: int, p_sel: float) -> None:
        p = self.position(q)
        if self._is_local(p):
            share = self.shard.collapse(p, bit) if self.w > 0 else 0.0
            self.w = self.w * math.sqrt(share / p_sel) if share > 0 else 0.0
            self.nl -= 1
        else:
            b = self._rank_bit(p)
            self.w = self.w / math.sqrt(p_sel) if ((self.rank >> b) & 1) == bit else 0.0
            self.frozen[b] = bit
            del self.rank_bits[p - self.nl]
        del self.perm[p]
        self.perm = [x - 1 if x > q else x for x in self.perm]
        self.n -= 1

    def reduced_density(self, keep: Sequence[int]) -> np.ndarray:
        """Reduced density matrix over the logical qubits `keep`, index bits
        in increasing qubit order (funmatrix.c:905-1037 evaluated for all
        elements): the kept qubits are swapped onto local positions, each
        rank contributes w_r^2 rho(v_r) and one all-reduce sums them."""
        keep = sorted(keep)
        if len(keep) > self.nl:
            raise ValueError("more kept qubits than local positions")
        for q in keep:
            p = self.position(q)
            if not self._is_local(p):
                self._swap_in(p, avoid=set(keep))
        self._flush()
        pos = [self.position(q) for q in keep]
        order = sorted(range(len(keep)), key=lambda i: pos[i])
        k = len(keep)
        dim = 1 << k
        if self.w > 0:
            rho = self.w * self.w * self.shard.reduced_density(sorted(pos))
        else:
            rho = np.zeros((dim, dim), dtype=np.complex128)
        # the shard's index bit j is the kept qubit at the j-th smallest
        # position; move it to that qubit's rank among `keep`
        idx = np.arange(dim)
        src = np.zeros(dim, dtype=np.int64)
        for j, i in enumerate(order):
            src |= ((idx >> i) & 1) << j
        rho = rho[np.ix_(src, src)]
        flat = self._allreduce(np.ascontiguousarray(rho).view(np.float64).reshape(-1))
        return flat.view(np.complex128).reshape(dim, dim)

    def gather(self) -> Optional[np.ndarray]:
        """The whole register in logical qubit order on rank 0 (None
        elsewhere): for checks on small registers."""
        self._flush()
        import torch
        local = self.shard.amplitudes() * self.w if self.w > 0 else \
            np.zeros(1 << self.nl, dtype=np.complex128)
        t = torch.from_numpy(np.ascontiguousarray(local, dtype=np.complex128).view(np.float64))
        if self.cuda_collectives:
            t = t.cuda()
        parts = [torch.zeros_like(t) for _ in range(self.world)]
        self.comm.all_gather(parts, t, group=self.group)
        parts = [x.cpu() for x in parts]
        if self.rank != 0:
            return None
        out = np.zeros(1 << self.n, dtype=np.complex128)
        for r in range(self.world):
            if any(((r >> b) & 1) != v for b, v in self.frozen.items()):
                continue
            amps = parts[r].numpy().view(np.complex128)
            j = np.arange(1 << self.nl)
            idx = np.zeros(1 << self.nl, dtype=np.int64)
            for p in range(self.nl):
                idx |= ((j >> p) & 1) << self.perm[p]
            for p in range(self.nl, self.n):
                b = self.rank_bits[p - self.nl]
                idx |= ((r >> b) & 1) << self.perm[p]
            out[idx] += amps
        return out
