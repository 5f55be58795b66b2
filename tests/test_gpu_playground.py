"""The reference playground's circuits (GHZ, QFT, IQFT, Grover, QAOA Max-Cut) on the
B200 path -- fused planner, NVRTC pass kernels, exact sampler -- against the oracle."""
import numpy as np
import pytest

import oracle_ffi as O
from quantumsimevo_b200 import playground as P
from quantumsimevo_b200.circuit import Circuit, Device

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def dev():
    return Device.default()


def _run(dev, n, ops, shots=3000, seed=0):
    c = Circuit(n, device=dev, seed=7)
    c.add_ops(ops)
    c.execute()
    st = c.get_state_vector()
    u = np.random.default_rng(seed).random(shots)
    got = c.sample(len(u), uniforms=u)
    assert np.array_equal(got, O.sample(st, n, u))     # sampler on the device state: exact
    return st


# tsp(): the 4-city distances of QSEplayground.cpp, two layers of the XY-mixer ansatz
_DIST4 = [[0, 3, 4, 2], [3, 0, 5, 7], [4, 5, 0, 6], [2, 7, 6, 0]]


def _tsp4_schedule():
    penalty, gammas, betas = P.tsp_schedule(-1.0, 1.0, 0.8, 0.4, 2, _DIST4)
    return penalty, 1.0, gammas, betas


CASES = [
    ("ghz", 16, lambda: P.ghz(16)),
    ("qft", 14, lambda: P.qft(14)),
    ("qft", 21, lambda: P.qft(21)),
    ("iqft", 14, lambda: P.iqft(14)),
    ("iqft", 21, lambda: P.iqft(21)),
    ("grover", 9, lambda: P.grover(300)),
    ("grover", 13, lambda: P.grover(5000)),
    ("maxcut", 14, lambda: P.qaoa_maxcut(14, [(i, (i + 1) % 14) for i in range(14)] +
                                         [(i, i + 7) for i in range(7)], [0.39, 0.81, 0.2], [1.05, 0.3, 0.7])),
    ("tsp", 16, lambda: P.tsp_xy_qaoa(_DIST4, *_tsp4_schedule())),
]


@pytest.mark.parametrize("name,n,build", CASES, ids=[f"{c[0]}{c[1]}" for c in CASES])
def test_playground_circuit_matches_oracle(dev, name, n, build):
    ops = build()
    st = _run(dev, n, ops)
    assert np.max(np.abs(st - O.run(n, ops))) <= TOL


def test_grover_finds_the_target(dev):
    target = 5000
    n, _ = P.grover_size(target)
    c = Circuit(n, device=dev, seed=3)
    c.add_ops(P.grover(target))
    c.execute()
    shots = c.sample(2000)
    assert np.mean(shots == target) > 0.95


@pytest.mark.parametrize("n,target,iterations", [(12, 3000, 300), (16, 40000, 120)])
def test_long_hadamard_runs_stay_finite(dev, n, target, iterations):
    # thousands of unscaled Hadamards inside one pass (12 qubits: one tile) and
    # across many passes (16 qubits): the pending 1/sqrt2 factors are applied
    # before the stored values can overflow
    ops = P.grover(target, iterations=iterations)
    assert P.grover_size(target)[0] == n
    st = _run(dev, n, ops, shots=1000)
    assert np.all(np.isfinite(st))
    assert np.max(np.abs(st - O.run(n, ops))) <= TOL
