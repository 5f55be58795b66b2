"""Fusion planner (host-only, no GPU): replaying every pass's gates in the
planned execution order on their planned physical qubits, then undoing the
final qubit relabelling, equals program order; every non-diagonal gate's
target sits in its pass's tile; every gate runs exactly once; and the
generated pass kernels compile for sm_100a (NVRTC runs without a GPU)."""
import ctypes as C
import json

import numpy as np
import pytest

import oracle_ffi as O
from quantumsimevo_b200 import _lib as L
from quantumsimevo_b200 import playground as P
from quantumsimevo_b200 import workloads as W

NONDIAG = {L.H, L.X, L.Y, L.RX, L.RY, L.GATE2X2, L.CNOT}
DIAG = {L.Z, L.PHASE, L.RZ, L.CPHASE, L.MCPHASE}


def describe(n, ops, k=0, max_gates=0, params=None):
    ops = np.ascontiguousarray(ops)
    need = C.c_size_t()
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
    pp = p.ctypes.data_as(C.POINTER(C.c_double)) if p is not None else None
    npar = 0 if p is None else p.size
    L.check(L.lib.qse_plan_describe(n, L.dptr(ops), len(ops), pp, npar, k, max_gates, None, 0, C.byref(need)))
    buf = C.create_string_buffer(need.value)
    L.check(L.lib.qse_plan_describe(n, L.dptr(ops), len(ops), pp, npar, k, max_gates, buf, need.value,
                                    C.byref(need)))
    return json.loads(buf.value.decode())


def dropped(op):
    t = int(op["type"])
    return t == L.IDENTITY or (t in (L.CNOT, L.SWAP) and int(op["target"]) == int(op["control"]))


def physical_op(op, pt, pc, psup):
    o = op.copy()
    t = int(op["type"])
    if t == L.CNOT:
        o["target"], o["control"] = pt, pc
    elif t == L.CPHASE:
        o["target"], o["control"] = pt, pc
    elif t == L.MCPHASE:
        o["target"] = pt
        o["controls"] = np.uint64(int(psup) & ~(1 << pt))
    else:
        o["target"] = pt
    return o


def check_plan(n, ops, k, max_gates=0):
    plan = describe(n, ops, k, max_gates)
    seen = []
    phys = []
    for p in plan["passes"]:
        tile = set(p["tile"])
        assert len(tile) == min(k, n)
        for src, pt, pc, psup in p["order"]:
            seen.append(src)
            t = int(ops[src]["type"])
            if t == L.SWAP:
                continue
            if t in NONDIAG and not dropped(ops[src]):
                assert pt in tile, (src, pt, tile)
            phys.append(physical_op(ops[src], pt, pc, psup))
        if max_gates:
            assert p["nondiag"] <= max_gates
    assert sorted(seen) == [i for i in range(len(ops)) if not dropped(ops[i])]
    want = O.run(n, ops)
    got_phys = O.run(n, W.to_array([tuple(o.tolist()) for o in phys])) if phys else O.run(n, ops[:0])
    perm = plan["perm"][:n]
    idx = np.arange(1 << n)
    pidx = np.zeros_like(idx)
    for q in range(n):
        pidx |= ((idx >> q) & 1) << perm[q]
    got = got_phys[pidx]
    assert np.max(np.abs(got - want)) < 1e-12
    return plan


@pytest.mark.parametrize("n,k", [(6, 4), (8, 5), (10, 6), (12, 8), (13, 9), (14, 12)])
def test_random_circuits_reorder_safely(n, k):
    for rep in range(4):
        ops = W.random_circuit(n, 150, 7000 + 13 * n + rep)
        check_plan(n, ops, k)


def test_gate_cap_respected():
    ops = W.random_circuit(12, 300, 99)
    check_plan(12, ops, 8, max_gates=5)


def test_qft_plan_is_few_passes_and_layouts():
    # 30-qubit H + RZ + QFT: 540 gates; the diagonal ladders never force a pass
    ops = W.hrz_qft(30, seed=2)
    plan = describe(30, ops, 12)
    assert len(plan["passes"]) <= 3
    assert sum(p["gates"] for p in plan["passes"]) == len(ops)
    # one register layout per block of 4 qubits that gets Hadamards
    assert max(p["layouts"] for p in plan["passes"]) <= 4
    check_plan(14, W.hrz_qft(14, seed=2), 6)


def test_playground_circuits_reorder_safely():
    # Grover's multi-controlled phases and X layers, the TSP XY mixer's H/RX-conjugated ZZ
    check_plan(10, P.grover(600, iterations=6), 8)
    dist = [[0, 2, 5], [2, 0, 3], [5, 3, 0]]
    penalty, gammas, betas = P.tsp_schedule(-1.0, 1.0, 0.8, 0.4, 2, dist)
    check_plan(9, P.tsp_xy_qaoa(dist, penalty, 1.0, gammas, betas), 6)


def test_swaps_are_relabels():
    n = 10
    ops = W.to_array([(L.SWAP, i, n - 1 - i, -1, 0, 0.0, 1.0, (0.0,) * 8) for i in range(n // 2)])
    plan = describe(n, ops, 8)
    perm = plan["perm"][:n]
    assert perm == list(reversed(range(n)))
    assert sum(p["nondiag"] for p in plan["passes"]) == 0


@pytest.mark.parametrize("name", ["qft16", "random12", "grover13", "tsp9", "qaoa12_adjoint"])
def test_generated_pass_kernels_compile(name):
    if name == "qft16":
        n, ops, params, ns = 16, W.hrz_qft(16, seed=2), None, 1
    elif name == "random12":
        n, ops, params, ns = 12, W.random_circuit(12, 200, 5), None, 1
    elif name == "grover13":
        # 71 iterations: many passes at the 256-gate cap, few distinct kernels
        n, ops, params, ns = 13, P.grover(5000), None, 1
    elif name == "tsp9":
        n, params, ns = 9, None, 1
        dist = [[0, 2, 5], [2, 0, 3], [5, 3, 0]]
        penalty, gammas, betas = P.tsp_schedule(-1.0, 1.0, 0.8, 0.4, 2, dist)
        ops = P.tsp_xy_qaoa(dist, penalty, 1.0, gammas, betas)
    else:
        ops, params, _, _ = W.qaoa_maxcut(12, 2, seed=3)
        n, ns = 12, 2
    size = C.c_size_t()
    p = None if params is None else np.ascontiguousarray(params)
    rc = L.lib.qse_plan_compile(n, L.dptr(ops), len(ops), p.ctypes.data_as(L._pd) if p is not None else None,
                                0 if p is None else p.size, 0, ns, C.byref(size))
    if rc == 6:
        pytest.skip("NVRTC not available: " + L.lib.qse_last_error().decode())
    L.check(rc)
    assert size.value > 0


@pytest.mark.parametrize("n,seed", [(26, 2), (30, 2)])
def test_streamed_pass_kernels_compile(n, seed):
    """The persistent streamed pass kernels (qse_plan_compile with nstates = 3:
    forward passes, streamed where a pass allows it) of the 26- and 30-qubit
    H + RZ + QFT circuits generate and compile for sm_100a."""
    ops = W.hrz_qft(n, seed=seed)
    size = C.c_size_t()
    rc = L.lib.qse_plan_compile(n, L.dptr(ops), len(ops), None, 0, 0, 3, C.byref(size))
    if rc == 6:
        pytest.skip("NVRTC not available: " + L.lib.qse_last_error().decode())
    L.check(rc)
    assert size.value > 0


@pytest.mark.parametrize("name", ["qft26", "qaoa24_adjoint"])
def test_precomputed_group_kernels_compile(name):
    """States of 22 qubits and more run their passes with the per-tile group
    values precomputed (no prologue in the pass kernel): forward passes of the
    26-qubit H + RZ + QFT circuit and adjoint reverse passes of 24-qubit QAOA
    generate and compile for sm_100a in that form."""
    if name == "qft26":
        n, ops, params, ns = 26, W.hrz_qft(26, seed=2), None, 1
    else:
        ops, params, _, _ = W.qaoa_maxcut(24, 2, seed=3)
        n, ns = 24, 2
    size = C.c_size_t()
    p = None if params is None else np.ascontiguousarray(params)
    rc = L.lib.qse_plan_compile(n, L.dptr(ops), len(ops), p.ctypes.data_as(L._pd) if p is not None else None,
                                0 if p is None else p.size, 0, ns, C.byref(size))
    if rc == 6:
        pytest.skip("NVRTC not available: " + L.lib.qse_last_error().decode())
    L.check(rc)
    assert size.value > 0
