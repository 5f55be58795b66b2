"""The context's plan cache: an execute of a program that ran before on a state
in the same layout reuses that plan, its kernels' sources and the compiled
kernels (engine.cu plan_for, compact_prefix).  The key holds every input the
plan depends on: the gates with their bound angles, the state's qubit map,
whether the state is a basis (or compact) state not yet written, the sampling
side output, the debug mode.  Every run below is compared bit for bit with the
same run on a new context (nothing cached), and the small ones with the oracle:
repeats, changed angles, changed qubit maps, more programs than the cache holds,
the compact route from different basis states, and a sampled state whose last
pass writes the probabilities."""
import ctypes as C

import numpy as np
import pytest

import oracle_ffi as O
from quantumsimevo_b200 import _lib as L
from quantumsimevo_b200 import workloads as W
from quantumsimevo_b200.circuit import Device, StateVector

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def dev():
    return Device.default()


def _execute(st, ops, params=None):
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
    pa = (p.ctypes.data_as(L._pd), p.size) if p is not None else (None, 0)
    L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), pa[0], pa[1], None, None, 0, None))


def _cold(n, runs):
    """The final state of `runs` ([(ops, params, reset_before)]) on a new context."""
    d = Device(0)
    st = StateVector(n, d)
    for ops, params, reset in runs:
        if reset:
            st.reset()
        _execute(st, ops, params)
    out = st.download()
    del st, d
    return out


def test_repeats_changed_angles_and_layouts(dev):
    n = 14
    a = W.random_circuit(n, 300, 1)
    b = np.concatenate([W.random_circuit(n, 200, 2), W.to_array(W.qft_ops(n))])   # ends in SWAPs
    q_ops, q_params, _, _ = W.qaoa_maxcut(n, 2, seed=3)
    st = StateVector(n, dev)
    seq = [(a, None, True), (b, None, True), (a, None, True), (a, None, True),
           (q_ops, q_params, True), (q_ops, q_params + 0.25, True), (q_ops, q_params, True),
           (b, None, False), (b, None, False), (a, None, False)]   # later ones start from relabelled states
    done = []
    for ops, params, reset in seq:
        if reset:
            st.reset()
        _execute(st, ops, params)
        done.append((ops, params, reset))
        got = st.download()
        assert np.array_equal(got, _cold(n, done[max(i for i, r in enumerate(done) if r[2]):]))
        if reset:
            assert np.max(np.abs(got - O.run(n, ops, params))) <= TOL


def test_more_programs_than_entries(dev):
    n = 12
    progs = [W.random_circuit(n, 120, 100 + s) for s in range(20)]
    st = StateVector(n, dev)
    for ops in progs + progs[:3]:
        st.reset()
        _execute(st, ops)
        assert np.max(np.abs(st.download() - O.run(n, ops))) <= TOL


def test_compact_route_from_different_basis_states(dev):
    n = 24
    ops = np.concatenate([W.random_circuit(12, 150, 5), W.random_circuit(22, 200, 6), W.random_circuit(n, 60, 7)])
    st = StateVector(n, dev)
    want0 = None
    for rep in range(3):
        st.reset()
        _execute(st, ops)
        got = st.download()
        if want0 is None:
            want0 = _cold(n, [(ops, None, True)])
        assert np.array_equal(got, want0)
    # from the basis state a measurement leaves (its bits on qubits the
    # compact prefix does not touch differ from |0..0>), then |0..0> again
    idx = C.c_uint64()
    L.check(L.lib.qse_measure(st.handle, 0.77, C.byref(idx)))
    _execute(st, ops)
    got = st.download()
    d = Device(0)
    ref = StateVector(n, d)
    _execute(ref, ops)
    L.check(L.lib.qse_measure(ref.handle, 0.77, C.byref(idx)))
    _execute(ref, ops)
    assert np.array_equal(got, ref.download())
    del ref, d
    st.reset()
    _execute(st, ops)
    assert np.array_equal(st.download(), want0)


def test_sampled_state_side_output(dev):
    """Executes alternating with samples: the later executes' last passes write
    the probabilities (a different kernel for the same gates); the outcomes equal
    those of a new context's first sample of the same state."""
    n = 22
    ops = np.concatenate([W.random_circuit(n, 200, 9), W.to_array(W.qft_ops(n))])
    u = np.random.default_rng(4).random(4000)
    st = StateVector(n, dev)
    outs = []
    for _ in range(4):
        st.reset()
        _execute(st, ops)
        out = np.empty(u.size, dtype=np.uint64)
        L.check(L.lib.qse_sample(st.handle, u.ctypes.data_as(L._pd), u.size, 0, out.ctypes.data_as(L._pu64)))
        outs.append(out)
    d = Device(0)
    ref = StateVector(n, d)
    _execute(ref, ops)
    want = np.empty(u.size, dtype=np.uint64)
    L.check(L.lib.qse_sample(ref.handle, u.ctypes.data_as(L._pd), u.size, 0, want.ctypes.data_as(L._pu64)))
    assert np.array_equal(st.download(), ref.download())
    del ref, d
    for out in outs:
        assert np.array_equal(out, want)
