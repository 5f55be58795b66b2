"""One state sharded over ranks (quantumsimevo_b200/sharded.py) on CPU: the
lowering (including X and Y on global qubits as relabellings), the half-shard
exchanges and the final qubit map, with the FP64 oracle as every shard's local
executor.  All shards in one process (LocalTransport) for 2 to 32 shards, and 2
and 4 gloo ranks in as many processes (TorchDistTransport)."""
import math
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import oracle_ffi as O
from quantumsimevo_b200 import _lib as L
from quantumsimevo_b200 import sharded as S
from quantumsimevo_b200 import workloads as W
from quantumsimevo_b200.workloads import _op, to_array

TOL = 1e-12


def _mixed(n, seed):
    """Every gate kind the lowering treats apart: global targets, global controls,
    multi-controlled phases across the global boundary, SWAPs, 2x2 gates."""
    ops = list(W.random_circuit(n, 30 * n, seed))
    rng = np.random.default_rng(seed)
    extra = []
    for _ in range(4 * n):
        a, b, c = rng.choice(n, 3, replace=False)
        th = float(rng.uniform(0, 2 * math.pi))
        extra += [_op(L.CNOT, int(a), int(b)), _op(L.RZ, int(a), theta=th), _op(L.CNOT, int(a), int(b)),
                  _op(L.MCPHASE, int(c), 0, th, (1 << int(a)) | (1 << int(b))),
                  _op(L.CPHASE, int(b), int(c), th), _op(L.Z, int(c)), _op(L.PHASE, int(a), theta=th),
                  _op(L.SWAP, int(a), int(c)), _op(L.H, int(b)),
                  _op(L.X, n - 1 - int(rng.integers(0, 3))), _op(L.Y, n - 1 - int(rng.integers(0, 3))),
                  _op(L.CNOT, n - 1, int(c))]
    return np.concatenate([np.asarray(ops, dtype=L.OP_DTYPE), to_array(extra)])


def _run_local(n, g, ops, params=None):
    nl = n - g
    shards = [np.zeros(1 << nl, dtype=np.complex128) for _ in range(1 << g)]
    shards[0][0] = 1.0
    progs, poss = [], []
    for r in range(1 << g):
        steps, pos = S.lower(ops, n, g, r, params)
        progs.append(steps)
        poss.append(pos)
    assert all(p == poss[0] for p in poss)
    tr = S.LocalTransport([torch.from_numpy(s) for s in shards])

    def execute(r, local_ops):
        shards[r][:] = O.run_on(shards[r], nl, local_ops)

    S.run_shards(progs, nl, execute, tr)
    return S.logical_order(shards, n, g, poss[0]), progs


@pytest.mark.parametrize("g", [1, 2, 3])
@pytest.mark.parametrize("seed", [1, 2])
def test_sharded_random_circuits_match_oracle(g, seed):
    n = 10
    ops = _mixed(n, 700 + seed)
    got, progs = _run_local(n, g, ops)
    assert np.max(np.abs(got - O.run(n, ops))) <= TOL
    assert any(st[0] == "exchange" for st in progs[0])


@pytest.mark.parametrize("seed", range(12))
def test_sharded_sweep_small_states(seed):
    # many small random circuits over 2 to 32 shards (down to two local qubits each)
    n = 7
    ops = _mixed(n, 900 + seed)
    want = O.run(n, ops)
    for g in (1, 2, 3, 5):
        got, _ = _run_local(n, g, ops)
        assert np.max(np.abs(got - want)) <= TOL


def test_sharded_qft_and_parameters():
    n, g = 11, 2
    ops = to_array(W.qft_ops(n))
    got, progs = _run_local(n, g, ops)
    assert np.max(np.abs(got - O.run(n, ops))) <= TOL
    # parameterised rotations bind as the engine binds them
    pops = to_array([_op(L.RY, q, param=q % 3, coeff=1.5, theta=0.1) for q in range(n)] +
                    [_op(L.RZ, q, param=(q + 1) % 3) for q in range(n)])
    params = np.array([0.3, -1.1, 2.4])
    got, _ = _run_local(n, g, pops, params)
    assert np.max(np.abs(got - O.run(n, pops, params))) <= TOL


def test_x_and_y_on_global_qubits_move_no_data():
    # qubits 6 and 7 stay global: X and Y on them, a CNOT and a phase controlled
    # by them, all without moving data until the relabelling left on qubit 7 is
    # resolved by the one exchange at the end
    n, g = 8, 2
    ops = to_array([_op(L.H, 0), _op(L.H, 1), _op(L.X, 7), _op(L.Y, 6), _op(L.CNOT, 2, 7),
                    _op(L.CPHASE, 0, 7, 0.4), _op(L.MCPHASE, 1, 0, 0.7, (1 << 6) | (1 << 7)),
                    _op(L.X, 6), _op(L.RZ, 6, theta=0.9), _op(L.Y, 7), _op(L.X, 7)])
    got, progs = _run_local(n, g, ops)
    assert np.max(np.abs(got - O.run(n, ops))) <= TOL
    assert sum(st[0] == "exchange" for st in progs[0]) == 1
    assert progs[0][-2][0] == "exchange"


def test_local_only_circuits_exchange_nothing():
    n, g = 9, 2
    ops = to_array([_op(L.H, q) for q in range(n - g)] + [_op(L.CPHASE, 0, n - 1, 0.7), _op(L.RZ, n - 2, theta=0.3),
                                                           _op(L.CNOT, 1, n - 1), _op(L.SWAP, 0, n - 1)])
    got, progs = _run_local(n, g, ops)
    assert np.max(np.abs(got - O.run(n, ops))) <= TOL
    assert not any(st[0] == "exchange" for st in progs[0])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, outdir, chunk_bytes=256 << 20):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import datetime

    import torch.distributed as dist
    import oracle_ffi as Ow
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        n, g = 10, world.bit_length() - 1
        nl = n - g
        ops = _mixed(n, 705)
        steps, pos = S.lower(ops, n, g, rank)
        shard = np.zeros(1 << nl, dtype=np.complex128)
        if rank == 0:
            shard[0] = 1.0
        tr = S.TorchDistTransport(torch.from_numpy(shard), rank, dist, chunk_bytes=chunk_bytes)

        def execute(local_ops):
            shard[:] = Ow.run_on(shard, nl, local_ops)

        S.run_rank(steps, nl, execute, tr)
        np.savez(os.path.join(outdir, f"r{rank}.npz"), shard=shard, pos=np.array(pos))
    finally:
        dist.destroy_process_group()


def test_exchange_pieces_cover_the_half_once():
    for rows, cols, chunk in [(1, 512, 512), (1, 512, 100), (8, 64, 64), (8, 64, 200), (16, 4, 3), (4, 16, 1),
                              (2, 1 << 20, 1 << 18)]:
        seen = np.zeros((rows, cols), dtype=np.int32)
        last = -1
        for r0, nr, c0, nc in S.exchange_pieces(rows, cols, chunk):
            assert 0 < nr * nc <= max(chunk, 1)
            seen[r0:r0 + nr, c0:c0 + nc] += 1
            assert r0 * cols + c0 > last      # address order
            last = r0 * cols + c0
        assert np.all(seen == 1), (rows, cols, chunk)


# chunk sizes: one piece per exchange (256 MiB), and pieces of 4 and 3 amplitudes
# (whole rows, cut rows, and ragged last pieces, each pipelined two deep)
@pytest.mark.parametrize("world,chunk_bytes", [(2, 256 << 20), (4, 256 << 20), (2, 64), (4, 48)])
def test_gloo_ranks_exchange_halves(tmp_path, world, chunk_bytes):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, str(tmp_path), chunk_bytes)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
        if p.is_alive():
            p.kill()
            pytest.fail("rank did not finish")
        assert p.exitcode == 0
    d = [np.load(tmp_path / f"r{r}.npz") for r in range(world)]
    assert all(np.array_equal(d[0]["pos"], x["pos"]) for x in d)
    n = 10
    got = S.logical_order([x["shard"] for x in d], n, world.bit_length() - 1, list(d[0]["pos"]))
    assert np.max(np.abs(got - O.run(n, _mixed(n, 705)))) <= TOL
