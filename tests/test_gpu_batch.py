"""Batched forward + adjoint (qse_batch_*) against the FP64 oracle's adjoint
(oracle/qse_oracle.c orc_adjoint, itself checked against parameter shift),
on every work-item shape the persistent kernel has: single-CTA circuits,
multi-tile circuits queued level-major behind completion counters, chains of
several tiles in one CTA, and both register layouts.  Also: graph replay with
new parameters, graph on/off and run-to-run determinism, device buffers,
autotune and its cache, empty circuits, argument errors.  Gradient tolerance
1e-10 (absolute), values 1e-10."""
import json

import numpy as np
import pytest

import oracle_ffi as O
from quantumsimevo_b200 import _lib as L
from quantumsimevo_b200 import workloads as W
from quantumsimevo_b200.batch import Batch, BatchConfig
from quantumsimevo_b200.circuit import Device

pytestmark = pytest.mark.gpu
TOL = 1e-10


@pytest.fixture(scope="module")
def dev():
    return Device.default()


def hea(count, wmin, wmax, dmin, dmax, seed):
    out = W.hea_batch(count, wmin, wmax, dmin, dmax, seed)
    circs = [(w, ops, len(p), obs) for (w, ops, p, obs) in out]
    params = np.concatenate([p for (_, _, p, _) in out])
    return circs, params


def mixed(count, wmin, wmax, seed):
    """Random circuits over every gate type, parameterised gates bound to a few
    shared parameters with random coefficients, multi-qubit Z-string observables."""
    rng = W.SplitMix64(seed)
    circs, params = [], []
    for c in range(count):
        n = wmin + rng.below(wmax - wmin + 1)
        ops = W.random_circuit(n, 40 + rng.below(60), seed * 1000 + c, with_2x2=True)
        npar = 1 + rng.below(6)
        for i in range(len(ops)):
            if int(ops[i]["type"]) in (L.RX, L.RY, L.RZ, L.PHASE, L.CPHASE, L.MCPHASE) and rng.below(4) != 0:
                ops[i]["param"] = rng.below(npar)
                ops[i]["coeff"] = rng.uniform() * 2.0 - 1.0
        z = [1 << q for q in range(n)] + [3, (1 << (n - 1)) | 1]
        wts = [rng.uniform() - 0.5 for _ in z]
        circs.append((n, ops, npar, (z, wts, rng.uniform())))
        params += [rng.uniform() * 6.28 for _ in range(npar)]
    return circs, np.array(params)


def oracle_all(circs, params):
    vals, grads, off = [], [], 0
    for (n, ops, npar, obs_t) in circs:
        obs, keep = L.observable(*obs_t)
        v, g = O.adjoint(n, ops, params[off:off + npar], obs)
        vals.append(v)
        grads.append(g)
        off += npar
    return np.array(vals), np.concatenate(grads) if grads else np.zeros(0)


def check(dev, circs, params, cfg=None, graph=True):
    b = Batch(circs, dev)
    if cfg is not None:
        b.config = cfg
    b.use_graph(graph)
    v, g = b.run(params)
    vw, gw = oracle_all(circs, params)
    assert np.max(np.abs(v - vw)) <= TOL
    if gw.size:
        assert np.max(np.abs(g - gw)) <= TOL
    return b, v, g


def test_single_cta_circuits(dev):
    circs, params = hea(24, 4, 11, 1, 5, seed=1)
    check(dev, circs, params)


def test_multi_tile_queue(dev):
    # 32 threads x 8 amplitudes: 8 tile qubits, circuits of 9..13 qubits span 2..32 tiles
    circs, params = hea(20, 6, 13, 2, 6, seed=2)
    check(dev, circs, params, BatchConfig(threads=32, reg_bits=3))


def test_multi_tile_two_register_bits(dev):
    circs, params = hea(16, 6, 12, 2, 5, seed=3)
    check(dev, circs, params, BatchConfig(threads=64, reg_bits=2))


def test_chains_of_tiles(dev):
    circs, params = hea(16, 6, 12, 2, 5, seed=4)
    check(dev, circs, params, BatchConfig(threads=32, reg_bits=3, chain_tiles=4))


def test_gate_cap_more_passes(dev):
    circs, params = hea(12, 8, 12, 3, 6, seed=5)
    check(dev, circs, params, BatchConfig(threads=64, reg_bits=3, max_gates=5))


@pytest.mark.parametrize("cfg", [None, BatchConfig(threads=32, reg_bits=3), BatchConfig(threads=32, reg_bits=2,
                                                                                         chain_tiles=2)])
def test_every_gate_type(dev, cfg):
    circs, params = mixed(14, 5, 11, seed=6)
    check(dev, circs, params, cfg)


def test_graph_off_same_bits_and_deterministic(dev):
    circs, params = hea(12, 6, 13, 2, 5, seed=7)
    cfg = BatchConfig(threads=32, reg_bits=3)
    b, v1, g1 = check(dev, circs, params, cfg, graph=True)
    v2, g2 = b.run(params)
    assert np.array_equal(v1, v2) and np.array_equal(g1, g2)
    b.use_graph(False)
    v3, g3 = b.run(params)
    assert np.array_equal(v1, v3) and np.array_equal(g1, g3)


def test_rebind_parameters_on_replay(dev):
    circs, params = hea(10, 5, 12, 2, 4, seed=8)
    b = Batch(circs, dev)
    b.config = BatchConfig(threads=64, reg_bits=3)
    b.run(params)
    rng = np.random.default_rng(9)
    for _ in range(2):
        p2 = rng.uniform(0, 2 * np.pi, params.size)
        v, g = b.run(p2)
        vw, gw = oracle_all(circs, p2)
        assert np.max(np.abs(v - vw)) <= TOL
        assert np.max(np.abs(g - gw)) <= TOL


def test_device_buffers(dev):
    torch = pytest.importorskip("torch")
    circs, params = hea(8, 5, 11, 2, 4, seed=10)
    b = Batch(circs, dev)
    p = torch.tensor(params, dtype=torch.float64, device="cuda:0")
    v = torch.zeros(len(circs), dtype=torch.float64, device="cuda:0")
    g = torch.zeros(params.size, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    b.run_device(p.data_ptr(), v.data_ptr(), g.data_ptr())
    dev.synchronize()
    vw, gw = oracle_all(circs, params)
    assert np.max(np.abs(v.cpu().numpy() - vw)) <= TOL
    assert np.max(np.abs(g.cpu().numpy() - gw)) <= TOL


def test_empty_and_parameter_free_circuits(dev):
    n = 6
    obs = ([1, 2, 4], [0.5, -1.0, 2.0], 0.25)
    fixed = W.random_circuit(n, 30, 11, with_2x2=True)
    circs = [(n, fixed[:0], 0, obs), (n, fixed, 0, obs), (7, W.hea_batch(1, 7, 7, 2, 2, 12)[0][1], 28,
                                                        ([1 << q for q in range(7)], [1.0] * 7, 0.0))]
    params = W.hea_batch(1, 7, 7, 2, 2, 12)[0][2]
    b = Batch(circs, dev)
    v, g = b.run(params)
    assert abs(v[0] - (0.25 + 0.5 - 1.0 + 2.0)) <= TOL
    vw, gw = oracle_all(circs, params)
    assert np.max(np.abs(v - vw)) <= TOL
    assert np.max(np.abs(g - gw)) <= TOL


def test_autotune_and_cache(dev, tmp_path):
    circs, params = hea(16, 6, 14, 2, 4, seed=13)
    b = Batch(circs, dev)
    b.run(params)
    path = tmp_path / "tune.json"
    cfg = b.autotune(str(path))
    data = json.loads(path.read_text())
    assert len(data) == 1
    (entry,) = data.values()
    assert entry["threads"] == cfg.threads and entry["reg_bits"] == cfg.reg_bits
    v, g = b.run(params)
    vw, gw = oracle_all(circs, params)
    assert np.max(np.abs(g - gw)) <= TOL
    b2 = Batch(circs, dev)
    assert b2.autotune(str(path)) == cfg  # served from the cache


def test_stats_and_errors(dev):
    circs, params = hea(6, 9, 12, 2, 3, seed=14)
    b = Batch(circs, dev)
    b.config = BatchConfig(threads=32, reg_bits=3)
    b.run(params)
    s = b.stats()
    assert s["passes"] > 0 and s["items"] > 0 and s["last_ms"] > 0 and s["hbm_bytes"] > 0
    with pytest.raises(L.QseError):
        b.config = BatchConfig(threads=48)
    with pytest.raises(L.QseError):
        b.config = BatchConfig(reg_bits=4)
    with pytest.raises(ValueError):
        b.run(params[:-1])
    bad = [(5, circs[0][1], circs[0][2], circs[0][3])]  # ops on qubits >= 5
    with pytest.raises(L.QseError):
        Batch(bad, dev).run(params[: circs[0][2]])


def test_hea_512_finite_differences(dev):
    """The full 512-circuit batch (widths 10..22, depths 4..12): every circuit's
    gradient against a central difference of the batch's own values, one shifted
    parameter per circuit (each value depends only on its own circuit's
    parameters), and the circuits of up to 13 qubits against the oracle."""
    circs, params = hea(512, 10, 22, 4, 12, seed=5)
    b = Batch(circs, dev)
    v, g = b.run(params)
    rng = np.random.default_rng(15)
    off = np.concatenate([[0], np.cumsum([c[2] for c in circs])])
    pick = np.array([off[i] + rng.integers(0, circs[i][2]) for i in range(len(circs))])
    h = 1e-5
    pp, pm = params.copy(), params.copy()
    pp[pick] += h
    pm[pick] -= h
    vp, _ = b.run(pp)
    vm, _ = b.run(pm)
    fd = (vp - vm) / (2 * h)
    assert np.max(np.abs(fd - g[pick])) <= 2e-6
    small = [i for i, c in enumerate(circs) if c[0] <= 13]
    assert small
    for i in small[:12]:
        obs, keep = L.observable(*circs[i][3])
        vw, gw = O.adjoint(circs[i][0], circs[i][1], params[off[i]:off[i + 1]], obs)
        assert abs(v[i] - vw) <= TOL
        assert np.max(np.abs(g[off[i]:off[i + 1]] - gw)) <= TOL


def test_bounded_wait_gives_up_and_batch_recovers(dev):
    """The persistent kernel's dependency waits are bounded.  With a limit of one
    poll, a dependent work item of a multi-tile queue finds its pass unfinished
    and gives up: it sets the error word, every CTA stops claiming work and
    leaves, and the run returns QSE_ERR_TIMEOUT -- no kernel keeps waiting and
    nothing faults.  The next run with the default limit matches the oracle."""
    circs, params = hea(4, 18, 18, 3, 3, seed=77)   # 18 qubits: 128 tiles per pass at the default tile
    b = Batch(circs, dev)
    b.set_wait_limit(1)
    gave_up = 0
    for _ in range(3):
        try:
            b.run(params)
        except L.QseError as e:
            assert e.status == 7, e   # QSE_ERR_TIMEOUT
            gave_up += 1
    assert gave_up >= 1
    b.set_wait_limit(0)
    v, g = b.run(params)
    vw, gw = oracle_all(circs, params)
    assert np.max(np.abs(v - vw)) <= TOL
    assert np.max(np.abs(g - gw)) <= TOL
