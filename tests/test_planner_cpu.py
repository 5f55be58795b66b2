"""Fusion planner (host-only, no GPU): the planned execution order applied
gate by gate with the oracle equals program order, every non-diagonal gate's
target sits in its pass's tile, and every gate runs exactly once."""
import ctypes as C
import json

import numpy as np
import pytest

import oracle_ffi as O
from quantumsimevo_b200 import _lib as L
from quantumsimevo_b200 import workloads as W

NONDIAG = {L.H, L.X, L.Y, L.RX, L.RY, L.GATE2X2, L.CNOT}


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


def check_plan(n, ops, k, max_gates=0):
    plan = describe(n, ops, k, max_gates)
    order = []
    for p in plan["passes"]:
        tile = set(p["tile"])
        assert len(tile) == min(k, n)
        for src, pt in p["order"]:
            order.append(src)
            if int(ops[src]["type"]) in NONDIAG and not dropped(ops[src]):
                assert pt in tile, (src, pt, tile)
        if max_gates:
            assert p["nondiag"] <= max_gates
    expect = [i for i in range(len(ops)) if not dropped(ops[i])]
    assert sorted(order) == expect
    want = O.run(n, ops)
    got = O.run(n, ops[order]) if order else O.run(n, ops[:0])
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


def test_qft_plan_is_few_passes():
    # 30-qubit H + RZ + QFT: 540 gates; the diagonal ladders never force a pass
    ops = W.hrz_qft(30, seed=2)
    plan = describe(30, ops, 12)
    assert len(plan["passes"]) <= 6
    assert sum(p["gates"] for p in plan["passes"]) == len(ops)
    # order check on a smaller instance with the same structure
    check_plan(14, W.hrz_qft(14, seed=2), 6)


def test_swaps_are_relabels():
    n = 10
    ops = W.to_array([(L.SWAP, i, n - 1 - i, -1, 0, 0.0, 1.0, (0.0,) * 8) for i in range(n // 2)])
    plan = describe(n, ops, 8)
    perm = plan["perm"][:n]
    assert perm == list(reversed(range(n)))
    assert sum(p["nondiag"] for p in plan["passes"]) == 0
