"""The playground circuit builders (quantumsimevo_b200/playground.py) against the
reference playground's own builders, compiled from its sources into oracle/_ref,
and against the oracle."""
import ctypes as C
import json
import math

import numpy as np
import pytest

import oracle_ffi as O
from quantumsimevo_b200 import _lib as L
from quantumsimevo_b200 import playground as P


@pytest.fixture(scope="module")
def ref():
    r = O.load_reference()
    if r is None:
        pytest.skip("oracle/_ref/libqse_ref_cpu.so not built")
    r.ref_set_quiet(1)
    return r


@pytest.mark.parametrize("which,n", [(0, 1), (0, 5), (0, 9), (1, 1), (1, 6), (1, 9)])
def test_qft_iqft_match_reference_builders(ref, which, n):
    ops = P.qft(n) if which == 0 else P.iqft(n)
    want = O.ref_playground(ref, which, n)
    # the same gates in the same order through the reference Circuit: identical arithmetic
    assert np.array_equal(O.ref_run(ref, n, ops), want)
    assert np.max(np.abs(O.run(n, ops) - want)) <= 1e-12


@pytest.mark.parametrize("target", [1, 5, 37, 200])
def test_grover_matches_reference_builder(ref, target):
    n, it = P.grover_size(target)
    want = O.ref_playground(ref, 2, n, target, it)
    ops = P.grover(target)
    assert np.array_equal(O.ref_run(ref, n, ops), want)
    assert np.max(np.abs(O.run(n, ops) - want)) <= 1e-12
    if n >= 6:
        assert abs(want[target]) ** 2 > 0.9      # the search finds the marked item


def test_grover_sizes_of_the_playground_targets():
    assert P.grover_size(29123321) == (25, 4550)   # round(4549.51)
    assert P.grover_size(802008535) == (30, 25736)
    assert P.grover_size(1) == (1, 1)
    zeros = 25 - bin(29123321).count("1")            # oracle X gates per side
    assert len(P.grover(29123321)) == 25 + 4550 * ((2 * zeros + 1) + (4 * 25 + 1))


def test_ghz_state():
    n = 9
    st = O.run(n, P.ghz(n))
    want = np.zeros(1 << n, dtype=np.complex128)
    want[0] = want[-1] = 1 / math.sqrt(2)
    assert np.max(np.abs(st - want)) <= 1e-15


def test_maxcut30_shape_and_angles():
    ops = P.maxcut30(3)
    assert len(ops) == 30 + 3 * (45 * 3 + 30)
    assert len(P.MAXCUT30_EDGES) == 45 and len(set(P.MAXCUT30_EDGES)) == 45
    rz = ops[ops["type"] == L.RZ]["theta"]
    rx = ops[ops["type"] == L.RX]["theta"]
    # QAOA.cpp:130,135: 4 * gamma[i] and 2 * beta[i] with float gamma, beta
    assert np.all(rz == float(np.float32(4) * np.float32(math.pi / 8)))
    assert np.all(rx == float(np.float32(2) * np.float32(math.pi / 3)))


def test_maxcut_small_against_reference_circuit(ref):
    # a 10-node ring with chords, p = 2, through the reference Circuit and the oracle
    n = 10
    edges = [(i, (i + 1) % n) for i in range(n)] + [(i, i + n // 2) for i in range(n // 2)]
    ops = P.qaoa_maxcut(n, edges, [0.3, 0.7], [0.9, 0.2])
    assert np.max(np.abs(O.run(n, ops) - O.ref_run(ref, n, ops))) <= 1e-12


def _passes(ops, n):
    need = C.c_size_t()
    L.check(L.lib.qse_plan_describe(n, L.dptr(ops), len(ops), None, 0, 12, 0, None, 0, C.byref(need)))
    buf = C.create_string_buffer(need.value)
    L.check(L.lib.qse_plan_describe(n, L.dptr(ops), len(ops), None, 0, 12, 0, buf, need.value, C.byref(need)))
    return len(json.loads(buf.value.decode())["passes"])


def test_grover_plan_is_linear_in_iterations():
    # planning stops scanning once every qubit is blocked: passes grow linearly
    a, b, c = (_passes(P.grover(29123321, iterations=it), 25) for it in (10, 20, 30))
    assert b - a == c - b > 0


def _ref_ising(ref, dist, penalty, weight, row, col):
    n = len(dist)
    d = np.ascontiguousarray(np.asarray(dist, dtype=np.float64).reshape(-1))
    h = np.zeros(n * n)
    cap = (n * n) ** 2
    pairs = (C.c_uint * (2 * cap))()
    coeffs = np.zeros(cap)
    cnt = C.c_uint()
    assert ref.ref_tsp_ising(d.ctypes.data_as(O._pd), n, penalty, weight, int(row), int(col),
                             h.ctypes.data_as(O._pd), pairs, coeffs.ctypes.data_as(O._pd), cap, C.byref(cnt)) == 0
    return h, {(pairs[2 * k], pairs[2 * k + 1]): coeffs[k] for k in range(cnt.value)}


@pytest.mark.parametrize("row,col", [(False, True), (True, True)])
def test_tsp_ising_matches_reference(ref, row, col):
    # the reference's own TVS::buildIsing: every field and coupling the same double
    penalty, _, _ = P.tsp_schedule(-1.0, 1.0, 0.8, 0.4, 4, P.TSP5_DIST)
    assert penalty == 36.0
    h_ref, j_ref = _ref_ising(ref, P.TSP5_DIST, penalty, 1.0, row, col)
    h, pairs, coeffs = P.tsp_ising(5, penalty, 1.0, P.TSP5_DIST, row, col)
    assert np.array_equal(np.array(h), h_ref)
    assert dict(zip(pairs, coeffs)) == j_ref


def test_tsp_circuit_stays_in_the_feasible_rows(ref):
    # 3 cities (9 qubits): the XY ring mixer keeps one excitation per city row
    dist = [[0, 2, 5], [2, 0, 3], [5, 3, 0]]
    penalty, gammas, betas = P.tsp_schedule(-1.0, 1.0, 0.8, 0.4, 2, dist)
    ops = P.tsp_xy_qaoa(dist, penalty, 1.0, gammas, betas)
    st = O.run(9, ops)
    assert np.max(np.abs(st - O.ref_run(ref, 9, ops))) <= 1e-12
    idx = np.arange(1 << 9)
    rows_ok = np.ones(1 << 9, dtype=bool)
    for v in range(3):
        w = sum(((idx >> P.tsp_index(v, t, 3)) & 1) for t in range(3))
        rows_ok &= w == 1
    assert abs(np.sum(np.abs(st[rows_ok]) ** 2) - 1.0) <= 1e-12


def test_tsp5_workload_shape():
    ops = P.tsp5()
    _, pairs, _ = P.tsp_ising(5, 36.0, 1.0, P.TSP5_DIST, False, True)
    assert len(ops) == 5 + 4 * (3 * len(pairs) + 25 + 25 * 14)
