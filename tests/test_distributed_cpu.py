"""The multi-rank path of batched circuits on CPU: world size 2 over "gloo",
one process per rank, each rank evaluating its shard (here with the FP64
oracle's adjoint, the GPU kernel's own checker) and the results gathered on
every rank.  Checks: the deterministic split covers every circuit once and is
balanced; the gathered values and gradients equal a single-process evaluation
bit for bit; the max-over-ranks timing reduction."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from quantumsimevo_b200 import distributed as D
from quantumsimevo_b200 import workloads as W


def _circuits():
    out = W.hea_batch(10, 4, 8, 1, 3, seed=21)
    circs = [(w, ops, len(p), obs) for (w, ops, p, obs) in out]
    params = np.concatenate([p for (_, _, p, _) in out])
    return circs, params


def _oracle_eval(circs, params, idx):
    import oracle_ffi as O
    from quantumsimevo_b200 import _lib as L
    off = D.param_offsets(circs)
    vals, grads = [], []
    for i in idx:
        n, ops, npar, obs_t = circs[i]
        obs, keep = L.observable(*obs_t)
        v, g = O.adjoint(n, ops, params[off[i]:off[i + 1]], obs)
        vals.append(v)
        grads.append(g)
    return np.array(vals), (np.concatenate(grads) if grads else np.zeros(0))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, outdir):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        circs, params = _circuits()
        idx = D.shard_for_rank(circs, rank, world)
        v, g = _oracle_eval(circs, params, idx)
        vals, grads = D.gather_results(circs, idx, v, g, dist)
        t = D.max_over_ranks(1.0 + rank, dist)
        np.savez(os.path.join(outdir, f"r{rank}.npz"), vals=vals, grads=grads, t=t, idx=np.array(idx))
    finally:
        dist.destroy_process_group()


def test_balanced_shards_cover_once():
    costs = [2.0 ** w for w in (10, 22, 14, 22, 11, 17, 20, 13, 22, 19)]
    for world in (1, 2, 3, 4):
        shards = D.balanced_shards(costs, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(costs)
        assert shards == D.balanced_shards(costs, world)  # deterministic


def test_two_ranks_gloo_match_single_process(tmp_path):
    circs, params = _circuits()
    want_v, want_g = _oracle_eval(circs, params, range(len(circs)))
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        if p.is_alive():
            p.kill()
            pytest.fail("rank did not finish")
        assert p.exitcode == 0
    shards = []
    for r in range(world):
        d = np.load(tmp_path / f"r{r}.npz")
        assert np.array_equal(d["vals"], want_v)
        assert np.array_equal(d["grads"], want_g)
        assert float(d["t"]) == 2.0
        shards.append(list(d["idx"]))
    assert sorted(shards[0] + shards[1]) == list(range(len(circs)))
    assert shards[0] and shards[1]
