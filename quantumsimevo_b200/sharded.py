"""One state vector sharded over 2^g ranks (one per GPU).

The physical qubits 0..n-g-1 are local: each rank holds the 2^(n-g)
amplitudes whose top g bits spell its rank.  The top g physical qubits are
global.  Gates lower per rank (``lower``):

- diagonal gates (Z, PHASE, RZ, CPHASE, MCPHASE) need no data from other
  ranks: a global qubit's bit is the rank's own bit, so each becomes a local
  gate, a per-rank scalar, or nothing;
- a CNOT whose control is global becomes X on its target on the ranks whose
  control bit is 1;
- SWAP only relabels (as in the single-state engine), and so do X and Y on a
  global qubit (they flip which ranks hold its 0 and 1; Y adds a per-rank
  phase); a relabelling left at the end is resolved by one exchange;
- a non-diagonal gate on a global qubit first exchanges that qubit with a
  local one: each rank trades the half of its shard whose local bit differs
  from its global bit with the partner rank that differs in that global bit
  (one send and one receive of 2^(n-g-1) amplitudes).  The local qubit given
  up is the one whose next non-diagonal use lies furthest ahead (ties: the
  highest position, so the exchanged halves are long contiguous runs).

Every rank derives the same exchange sequence from the same op list, so the
ranks take the same collective steps in the same order.  Between exchanges a
rank runs its local ops through the single-GPU engine (fused passes), and
per-rank scalars are folded into one diagonal 2x2 gate on local qubit 0 (it
joins the next fused pass) before each exchange and at the end.

Transports: ``TorchDistTransport`` (torch.distributed point-to-point: NCCL
between GPUs, gloo on CPU) and ``LocalTransport`` (every shard in one
process, exchanges as copies).
"""
from __future__ import annotations

import cmath

import numpy as np

from . import _lib as L

_NONDIAG = (L.H, L.X, L.Y, L.RX, L.RY, L.GATE2X2)
_DIAG = (L.Z, L.PHASE, L.RZ, L.CPHASE, L.MCPHASE)


def _angle(op, params):
    """The engine's binding (engine.cu, bound_angle): theta + coeff * params[param]."""
    if int(op["param"]) < 0:
        return float(op["theta"])
    if params is None or int(op["param"]) >= len(params):
        raise ValueError("op parameter index out of range")
    return float(op["theta"]) + float(op["coeff"]) * float(params[int(op["param"])])


def _mk(t, target=0, control=0, theta=0.0, controls=0, m=None):
    return (t, target, control, -1, controls, theta, 1.0, tuple(m) if m is not None else (0.0,) * 8)


def lower(ops, n: int, g: int, rank: int, params=None):
    """Per-rank program of `ops` on an n-qubit state with g global qubits.
    Returns (steps, pos): steps is a list of ("ops", op array for the local
    (n-g)-qubit shard) and ("exchange", j, l) = swap global qubit n-g+j with
    local qubit l; pos[q] is logical qubit q's final physical position."""
    ops = L.as_ops(ops)
    nl = n - g
    if g < 0 or nl < 1:
        raise ValueError("need at least one local qubit")
    pos = list(range(n))
    where = list(range(n))
    flip = [0] * g          # X on a global qubit relabels: its value on rank r is bit j of r XOR flip[j]
    steps, pending = [], []
    scalar = [1.0 + 0.0j]

    def flush_scalar():
        s = scalar[0]
        if s != 1.0:
            pending.append(_mk(L.GATE2X2, 0, m=(s.real, s.imag, 0.0, 0.0, 0.0, 0.0, s.real, s.imag)))
            scalar[0] = 1.0 + 0.0j

    def flush_ops():
        # one op step per segment on every rank (possibly empty), so the
        # programs of all ranks line up step for step
        steps.append(("ops", L.as_ops(pending)))
        pending.clear()

    def gbit(q):
        p = pos[q]
        return None if p < nl else ((rank >> (p - nl)) & 1) ^ flip[p - nl]

    def exchange(j, lp):
        # global position nl + j <-> local position lp; a flipped global qubit
        # arrives holding the rank's bit, so one local X restores its value
        flush_scalar()
        flush_ops()
        steps.append(("exchange", j, lp))
        qg, ql = where[nl + j], where[lp]
        pos[qg], pos[ql] = lp, nl + j
        where[lp], where[nl + j] = qg, ql
        if flip[j]:
            pending.append(_mk(L.X, lp))
            flip[j] = 0

    types = ops["type"].astype(np.int64)
    targets = ops["target"].astype(np.int64)
    nondiag = np.isin(types, list(_NONDIAG) + [L.CNOT])

    def next_uses(i):
        # index of each qubit's next non-diagonal use at or after op i (one scan)
        nu = {}
        for k in np.nonzero(nondiag[i:])[0]:
            q = int(targets[i + k])
            if q not in nu:
                nu[q] = i + int(k)
                if len(nu) == n:
                    break
        return nu

    for i, op in enumerate(ops):
        t = int(op["type"])
        tq = int(op["target"])
        if t == L.IDENTITY:
            continue
        if t == L.SWAP:
            a, b = tq, int(op["control"])
            pos[a], pos[b] = pos[b], pos[a]
            where[pos[a]], where[pos[b]] = a, b
            continue
        if t in (L.X, L.Y) and pos[tq] >= nl:
            # X and Y on a global qubit move no data: flip which ranks hold 0 and 1
            j = pos[tq] - nl
            flip[j] ^= 1
            if t == L.Y:                  # Y|v> = i (-1)^v |1-v>: a phase by the new value
                scalar[0] *= 1j if gbit(tq) == 1 else -1j
            continue
        if t in _NONDIAG or t == L.CNOT:
            if pos[tq] >= nl:
                nu = next_uses(i)
                best = max(range(nl), key=lambda lp: (nu.get(where[lp], len(ops) + 1), lp))
                exchange(pos[tq] - nl, best)
            if t == L.CNOT:
                cv = gbit(int(op["control"]))
                if cv is None:
                    pending.append(_mk(L.CNOT, pos[tq], pos[int(op["control"])]))
                elif cv == 1:
                    pending.append(_mk(L.X, pos[tq]))
            elif t in (L.RX, L.RY):
                pending.append(_mk(t, pos[tq], theta=_angle(op, params)))
            elif t == L.GATE2X2:
                pending.append(_mk(t, pos[tq], m=op["m"]))
            else:
                pending.append(_mk(t, pos[tq]))
            continue
        if t not in _DIAG:
            raise ValueError(f"gate type {t} is not supported on a sharded state")
        th = _angle(op, params) if t != L.Z else 0.0
        if t in (L.Z, L.PHASE, L.RZ):
            v = gbit(tq)
            if v is None:
                pending.append(_mk(t, pos[tq], theta=th))
            elif t == L.RZ:
                scalar[0] *= cmath.exp(1j * (th / 2.0 if v else -th / 2.0))
            elif v:
                scalar[0] *= -1.0 if t == L.Z else cmath.exp(1j * th)
            continue
        if t == L.CPHASE:
            qs = [tq, int(op["control"])]
        else:
            cm = int(op["controls"])
            qs = [q for q in range(64) if (cm >> q) & 1 and q != tq] + [tq]
        if any(gbit(q) == 0 for q in qs):
            continue                      # a global bit is 0 on this rank: identity
        loc = [pos[q] for q in qs if gbit(q) is None]
        if not loc:
            scalar[0] *= cmath.exp(1j * th)
        elif len(loc) == 1:
            pending.append(_mk(L.PHASE, loc[0], theta=th))
        elif len(loc) == 2:
            pending.append(_mk(L.CPHASE, loc[0], loc[1], theta=th))
        else:
            mask = 0
            for p in loc[:-1]:
                mask |= 1 << p
            pending.append(_mk(L.MCPHASE, loc[-1], 0, theta=th, controls=mask))
    for j in range(g):
        if flip[j]:                       # leave no relabelling behind: the shards hold the state
            exchange(j, nl - 1)
    flush_scalar()
    flush_ops()
    return steps, pos


def logical_order(shards, n: int, g: int, pos) -> np.ndarray:
    """The full logical state from the shards (rank r's shard = physical indices
    r * 2^(n-g) ... ): amplitude of logical index x sits at physical index
    sum over q of bit q of x at position pos[q]."""
    phys = np.concatenate([np.asarray(s) for s in shards])
    idx = np.arange(1 << n, dtype=np.int64)
    p = np.zeros_like(idx)
    for q in range(n):
        p |= ((idx >> q) & 1) << pos[q]
    return phys[p]


class LocalTransport:
    """Every shard in this process (complex128 torch tensors on one device or on
    the host); an exchange swaps the halves between each pair of shards."""

    def __init__(self, tensors):
        self.t = tensors

    def exchange(self, j: int, l: int, nl: int):
        for r in range(len(self.t)):
            if (r >> j) & 1:
                continue
            a = self.t[r].view(1 << (nl - l - 1), 2, 1 << l)
            b = self.t[r | (1 << j)].view(1 << (nl - l - 1), 2, 1 << l)
            tmp = a[:, 1, :].clone()
            a[:, 1, :] = b[:, 0, :]
            b[:, 0, :] = tmp


class TorchDistTransport:
    """One shard per rank (a complex128 torch tensor); the exchange is a send and a
    receive of half the shard with the partner rank over torch.distributed (NCCL
    between GPUs, gloo on CPU), carried as float64 pairs so every backend takes it."""

    def __init__(self, tensor, rank: int, dist, group=None):
        self.t = tensor
        self.rank = rank
        self.dist = dist
        self.group = group

    def exchange(self, j: int, l: int, nl: int):
        import torch
        b = (self.rank >> j) & 1
        partner = self.rank ^ (1 << j)
        x = self.t.view(1 << (nl - l - 1), 2, 1 << l)
        send = torch.view_as_real(x[:, 1 - b, :].contiguous())
        recv = torch.empty_like(send)
        # one grouped send+receive: under NCCL both partners' sends and receives
        # are posted together (a send issued alone would wait for a receive that
        # sits queued behind the partner's own send on the same stream)
        ops = [self.dist.P2POp(self.dist.isend, send, partner, group=self.group),
               self.dist.P2POp(self.dist.irecv, recv, partner, group=self.group)]
        for rq in self.dist.batch_isend_irecv(ops):
            rq.wait()
        x[:, 1 - b, :] = torch.view_as_complex(recv)


def run_rank(steps, nl: int, execute, transport):
    """Runs one rank's lowered program: execute(ops) on its shard between the
    exchanges."""
    for st in steps:
        if st[0] == "ops":
            if len(st[1]):
                execute(st[1])
        else:
            transport.exchange(st[1], st[2], nl)


def run_shards(programs, nl: int, execute, transport):
    """Runs the lowered programs of every shard held in this process in lockstep:
    execute(r, ops) per shard, one transport.exchange per exchange step."""
    kinds = [[st[0] if st[0] == "ops" else st for st in p] for p in programs]
    if any(k != kinds[0] for k in kinds):
        raise RuntimeError("ranks lowered to different exchange sequences")
    for k in range(len(programs[0])):
        st = programs[0][k]
        if st[0] == "ops":
            for r, p in enumerate(programs):
                if len(p[k][1]):
                    execute(r, p[k][1])
        else:
            transport.exchange(st[1], st[2], nl)


class _DeviceArray:
    """CUDA array interface over the engine's device amplitudes (no copy)."""

    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (2 * count,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 2}


class DeviceShard:
    """One rank's shard: a state of n-g qubits in the single-GPU engine (fused
    passes for the local ops) with a torch view of its amplitudes for the
    exchanges.  Rank 0 starts in |0..0>, every other rank at zero."""

    def __init__(self, nl: int, rank: int, device=None):
        import torch
        from .circuit import Device, StateVector
        self.device = device or Device.default()
        self.nl = nl
        self.sv = StateVector(nl, self.device)
        self.torch_device = torch.device("cuda", self.device.index)
        if rank != 0:
            self.tensor().zero_()
            torch.cuda.synchronize(self.torch_device)

    def tensor(self):
        import torch
        p = L.C.c_void_p()
        L.check(L.lib.qse_state_device_ptr(self.sv.handle, L.C.byref(p)))
        t = torch.as_tensor(_DeviceArray(p.value, 1 << self.nl), device=self.torch_device)
        return torch.view_as_complex(t.view(-1, 2))

    def execute(self, ops):
        ops = np.ascontiguousarray(ops)
        L.check(L.lib.qse_execute(self.sv.handle, L.dptr(ops), len(ops), None, 0, None, None, 0, None))

    def synchronize(self):
        self.device.synchronize()

    def download(self) -> np.ndarray:
        return self.sv.download()


class _Synced:
    """Wraps a transport: the engine's stream finishes before an exchange, the
    exchange's torch work finishes before the engine's next launch."""

    def __init__(self, inner, shards):
        self.inner = inner
        self.shards = shards

    def exchange(self, j, l, nl):
        import torch
        for s in self.shards:
            s.synchronize()
        self.inner.exchange(j, l, nl)
        for s in self.shards:
            torch.cuda.synchronize(s.torch_device)


def execute_rank(ops, n: int, g: int, rank: int, shard: DeviceShard, dist, params=None, group=None):
    """This rank's part of executing ops on the sharded n-qubit state (one
    process per GPU, torch.distributed already initialised; NCCL between
    GPUs).  Returns the final logical -> physical qubit map."""
    steps, pos = lower(ops, n, g, rank, params)
    tr = _Synced(TorchDistTransport(shard.tensor(), rank, dist, group), [shard])
    run_rank(steps, n - g, shard.execute, tr)
    shard.synchronize()
    return pos


def execute_shards(ops, n: int, g: int, shards, params=None):
    """Every shard in this process (one GPU holding 2^g shards, or a test):
    the same lowering and exchanges as execute_rank, the exchanges as device
    copies.  Returns the final logical -> physical qubit map."""
    progs, pos = [], None
    for r in range(len(shards)):
        steps, pos = lower(ops, n, g, r, params)
        progs.append(steps)
    tr = _Synced(LocalTransport([s.tensor() for s in shards]), shards)
    run_shards(progs, n - g, lambda r, o: shards[r].execute(o), tr)
    for s in shards:
        s.synchronize()
    return pos
