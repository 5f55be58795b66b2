"""The pass kernels' debug mode: with QSE_DEBUG_BOUNDS set when a kernel is
generated, every global access it makes checks its index against the size of
its array (state, second state, compact input, probability output, block sums,
group-value table); an index outside would record status 8, which the next
synchronising call reports, and the access would be skipped.  These runs go
through the generated kernels of every input and output kind in that mode and
must report nothing and give the same bits as the normal kernels."""
import ctypes as C

import numpy as np
import pytest

import oracle_ffi as O
from quantumsimevo_b200 import _lib as L
from quantumsimevo_b200 import workloads as W
from quantumsimevo_b200.circuit import Device, StateVector

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    return Device.default()


def _run(dev, n, ops, shots=0, params=None):
    """State after ops from |0..0> (and, with shots, the outcomes of two samples
    with an execute between them, so the second reads the last pass's output)."""
    st = StateVector(n, dev)
    p = None if params is None else np.ascontiguousarray(params)
    pa = (p.ctypes.data_as(L._pd), p.size) if p is not None else (None, 0)

    def execute():
        L.check(L.lib.qse_state_reset(st.handle))
        L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), pa[0], pa[1], None, None, 0, None))

    execute()
    outs = []
    if shots:
        u = np.random.default_rng(n).random(shots)
        for _ in range(2):
            out = np.empty(shots, dtype=np.uint64)
            L.check(L.lib.qse_sample(st.handle, u.ctypes.data_as(L._pd), shots, 0, out.ctypes.data_as(L._pu64)))
            outs.append(out)
            execute()
    return st.download(), outs


@pytest.mark.parametrize("case", ["random13", "hrz_qft26", "relabel22"])
def test_debug_mode_kernels_report_nothing_and_match(dev, monkeypatch, case):
    if case == "random13":
        n, ops, shots = 13, W.random_circuit(13, 300, 5), 0
    elif case == "hrz_qft26":     # compact prefix, compact input, probability side output
        n, ops, shots = 26, W.hrz_qft(26, seed=2), 5000
    else:                         # relabelled qubits, precomputed group values, side output
        n, ops, shots = 22, np.concatenate([W.random_circuit(22, 200, 9), W.to_array(W.qft_ops(22))]), 5000
    want, want_out = _run(dev, n, ops, shots)
    monkeypatch.setenv("QSE_DEBUG_BOUNDS", "1")
    got, got_out = _run(dev, n, ops, shots)
    assert np.array_equal(got, want)
    for a, b in zip(got_out, want_out):
        assert np.array_equal(a, b)
    if case == "random13":
        assert np.max(np.abs(got - O.run(n, ops))) <= 1e-12


def test_debug_mode_adjoint_matches(dev, monkeypatch):
    n = 12
    ops, params, edges, obs_t = W.qaoa_maxcut(n, 2, seed=3)
    obs, keep = L.observable(*obs_t)

    def adjoint():
        st = StateVector(n, dev)
        p = np.ascontiguousarray(params)
        g = np.zeros(p.size)
        v = C.c_double()
        L.check(L.lib.qse_adjoint(st.handle, L.dptr(ops), len(ops), p.ctypes.data_as(L._pd), p.size, C.byref(obs),
                                  C.byref(v), g.ctypes.data_as(L._pd)))
        return v.value, g

    v0, g0 = adjoint()
    monkeypatch.setenv("QSE_DEBUG_BOUNDS", "1")
    v1, g1 = adjoint()
    assert v1 == v0 and np.array_equal(g1, g0)
