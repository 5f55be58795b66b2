"""Many circuits on many GPUs: one process per GPU (torch.distributed), the
circuits of a batch split across ranks with no collective on the data path,
results gathered once at the end.

A single state vector does not shard here (that would need an exchange step per
gate on a "global" qubit); independent circuits and parameter-shift
evaluations do.  Works with the "nccl" backend on GPUs and "gloo" on CPU (the
tests run the latter).
"""
from __future__ import annotations

import heapq

import numpy as np


def circuit_cost(nqubits: int, nops: int) -> float:
    """Work estimate of one forward + adjoint evaluation: amplitudes x gates."""
    return float(2 ** int(nqubits)) * max(1, int(nops))


def balanced_shards(costs, world: int):
    """Deterministic longest-processing-time split of items with the given costs
    into `world` lists of indices (each list ascending).  Every rank computes
    the same split from the same inputs, so no communication is needed."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    shards = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shards]


def shard_for_rank(circuits, rank: int, world: int):
    """Indices of the circuits (nqubits, ops, nparams, obs) this rank evaluates."""
    costs = [circuit_cost(c[0], len(c[1])) for c in circuits]
    return balanced_shards(costs, world)[rank]


def param_offsets(circuits):
    return np.concatenate([[0], np.cumsum([int(c[2]) for c in circuits])]).astype(np.int64)


def local_params(circuits, params, idx):
    """The concatenated parameters of the circuits idx (in idx order)."""
    off = param_offsets(circuits)
    return np.concatenate([params[off[i]:off[i + 1]] for i in idx]) if len(idx) else np.zeros(0)


def gather_results(circuits, idx, values, grads, dist, group=None):
    """Every rank passes the values / gradients of its circuits idx (in idx
    order); every rank gets the full arrays back, in circuit order."""
    payload = (list(map(int, idx)), np.asarray(values, dtype=np.float64), np.asarray(grads, dtype=np.float64))
    world = dist.get_world_size(group)
    parts = [None] * world
    dist.all_gather_object(parts, payload, group=group)
    off = param_offsets(circuits)
    all_values = np.zeros(len(circuits))
    all_grads = np.zeros(int(off[-1]))
    seen = np.zeros(len(circuits), dtype=bool)
    for ids, v, g in parts:
        pos = 0
        for k, i in enumerate(ids):
            if seen[i]:
                raise RuntimeError(f"circuit {i} evaluated by two ranks")
            seen[i] = True
            all_values[i] = v[k]
            npar = int(off[i + 1] - off[i])
            all_grads[off[i]:off[i + 1]] = g[pos:pos + npar]
            pos += npar
    if not seen.all():
        raise RuntimeError("some circuits were evaluated by no rank")
    return all_values, all_grads


def max_over_ranks(x: float, dist, device=None, group=None) -> float:
    """Max of a per-rank scalar (timings are reported as the slowest rank)."""
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
