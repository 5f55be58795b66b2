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


def exchange_pieces(rows: int, cols: int, chunk: int):
    """The exchanged half (rows x cols amplitudes, rows of cols contiguous
    amplitudes) cut into pieces of at most `chunk` amplitudes, in address
    order: (row0, nrows, col0, ncols).  Whole rows go together while a row fits
    in a chunk; longer rows are cut.  Both partners derive the same pieces."""
    chunk = max(1, chunk)
    if cols <= chunk:
        per = chunk // cols
        return [(r, min(per, rows - r), 0, cols) for r in range(0, rows, per)]
    return [(r, 1, c, min(chunk, cols - c)) for r in range(rows) for c in range(0, cols, chunk)]


class TorchDistTransport:
    """One shard per rank (a complex128 torch tensor); the exchange is a send and a
    receive of half the shard with the partner rank over torch.distributed (NCCL
    between GPUs, gloo on CPU), carried as float64 pairs so every backend takes it.

    The half travels in pieces of at most `chunk_bytes`, pipelined: piece k+1 is
    packed (when it is not one contiguous run) and posted before piece k is
    waited for and copied into place, so under NCCL the transfer of one piece
    overlaps the local copies of its neighbours on the compute stream, and the
    staging memory is four pieces instead of two half-shards.  A piece's place
    is overwritten only after its own send completed (its wait precedes the
    copy), and the buffers of piece k are reused by piece k+2 only after piece
    k's copy, which follows its wait."""

    def __init__(self, tensor, rank: int, dist, group=None, chunk_bytes: int = 256 << 20):
        self.t = tensor
        self.rank = rank
        self.dist = dist
        self.group = group
        self.chunk = max(1, chunk_bytes // 16)
        self._send = [None, None]
        self._recv = [None, None]

    def _buf(self, which, slot, n):
        import torch
        bufs = self._send if which == 0 else self._recv
        if bufs[slot] is None or bufs[slot].numel() < n:
            bufs[slot] = torch.empty(min(self.chunk, self.t.numel()), dtype=self.t.dtype, device=self.t.device)
        return bufs[slot][:n]

    def exchange(self, j: int, l: int, nl: int):
        import torch
        b = (self.rank >> j) & 1
        partner = self.rank ^ (1 << j)
        rows, cols = 1 << (nl - l - 1), 1 << l
        half = self.t.view(rows, 2, cols)[:, 1 - b, :]
        pieces = exchange_pieces(rows, cols, self.chunk)

        def view(k):
            r0, nr, c0, nc = pieces[k]
            return half[r0:r0 + nr, c0:c0 + nc]

        def post(k):
            src = view(k)
            n = src.numel()
            if src.is_contiguous():
                s = src.reshape(-1)
            else:
                s = self._buf(0, k & 1, n)
                s.view(src.shape).copy_(src)
            r = self._buf(1, k & 1, n)
            # one grouped send+receive: under NCCL both partners' sends and
            # receives are posted together (a send issued alone would wait for
            # a receive that sits queued behind the partner's own send)
            ops = [self.dist.P2POp(self.dist.isend, torch.view_as_real(s), partner, group=self.group),
                   self.dist.P2POp(self.dist.irecv, torch.view_as_real(r), partner, group=self.group)]
            return self.dist.batch_isend_irecv(ops), r

        pending = post(0)
        for k in range(len(pieces)):
            nxt = post(k + 1) if k + 1 < len(pieces) else None
            reqs, r = pending
            for rq in reqs:
                rq.wait()
            dst = view(k)
            dst.copy_(r.view(dst.shape))
            pending = nxt


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
        self.rank = rank
        self.sv = StateVector(nl, self.device)
        self.torch_device = torch.device("cuda", self.device.index)
        self.reset()

    def reset(self):
        """The shard of |0..0>: rank 0 holds |0..0> of its local qubits (recorded,
        not written: the next execute's first pass generates it), every other
        rank zeros."""
        import torch
        if self.rank == 0:
            L.check(L.lib.qse_state_reset(self.sv.handle))
        else:
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
    exchange's torch work finishes before the engine's next launch.  The
    transport is built at the first exchange (a shard's device view writes a
    recorded |0..0> out, which an execute with no exchange never needs).
    stats, if given, accumulates "exchanges", "exchange_s" (host wall time
    between the two synchronisations) and "exchange_bytes" (sent per rank)."""

    def __init__(self, make_inner, shards, stats=None):
        self.make_inner = make_inner
        self.inner = None
        self.shards = shards
        self.stats = stats

    def exchange(self, j, l, nl):
        import time

        import torch
        if self.inner is None:
            self.inner = self.make_inner()
        for s in self.shards:
            s.synchronize()
        t0 = time.perf_counter()
        self.inner.exchange(j, l, nl)
        for s in self.shards:
            torch.cuda.synchronize(s.torch_device)
        if self.stats is not None:
            self.stats["exchanges"] = self.stats.get("exchanges", 0) + 1
            self.stats["exchange_s"] = self.stats.get("exchange_s", 0.0) + time.perf_counter() - t0
            self.stats["exchange_bytes"] = self.stats.get("exchange_bytes", 0) + 8 * (1 << nl)


def execute_rank(ops, n: int, g: int, rank: int, shard: DeviceShard, dist, params=None, group=None, stats=None,
                 chunk_bytes: int = 256 << 20):
    """This rank's part of executing ops on the sharded n-qubit state (one
    process per GPU, torch.distributed already initialised; NCCL between
    GPUs).  Returns the final logical -> physical qubit map.  stats: see
    _Synced; chunk_bytes: the exchange's piece size (TorchDistTransport)."""
    steps, pos = lower(ops, n, g, rank, params)
    tr = _Synced(lambda: TorchDistTransport(shard.tensor(), rank, dist, group, chunk_bytes), [shard], stats)
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
    tr = _Synced(lambda: LocalTransport([s.tensor() for s in shards]), shards)
    run_shards(progs, n - g, lambda r, o: shards[r].execute(o), tr)
    for s in shards:
        s.synchronize()
    return pos
