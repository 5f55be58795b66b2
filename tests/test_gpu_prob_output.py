"""Probabilities written by the last pass of an execute.

Once a state has been sampled, the last pass of each later execute also
writes the probabilities |a|^2 of the amplitudes it stores, in logical order,
and (where a warp's values fall in one 4096-block) the block sums the
sampler's binade guess reads, so the next sample skips its gather over the
state.  An execute that finds the previous side output unread stops writing
it.  Every sample here is compared bit for bit with the oracle's sampler on
the downloaded state.
"""
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


def _execute(st, ops):
    L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, None, None, 0, None))


def _sample(st, u):
    out = np.empty(len(u), dtype=np.uint64)
    L.check(L.lib.qse_sample(st.handle, u.ctypes.data_as(L._pd), len(u), 0, out.ctypes.data_as(L._pu64)))
    return out


def _circuit(kind, n, seed):
    if kind == "swaps":          # relabelled qubits: the side output is a gather by the final map
        return W.random_circuit(n, 12 * n, seed)
    if kind == "identity":       # no SWAP: the logical order is the physical one
        return W.random_circuit(n, 12 * n, seed, types=[L.H, L.RX, L.RY, L.RZ, L.CNOT, L.CPHASE, L.PHASE])
    return W.hrz_qft(n, seed=seed)   # compact prefix, then one full-state pass with the side output


@pytest.mark.parametrize("kind,n", [("identity", 16), ("swaps", 20), ("identity", 22), ("hrz_qft", 26)])
def test_second_execute_feeds_the_sampler(dev, kind, n):
    st = StateVector(n, dev)
    rng = np.random.default_rng(n)
    _execute(st, _circuit(kind, n, 1))
    u1 = rng.random(2000)
    assert np.array_equal(_sample(st, u1), O.sample(st.download(), n, u1))   # turns the side output on
    L.check(L.lib.qse_state_reset(st.handle))
    _execute(st, _circuit(kind, n, 2))
    u2 = rng.random(20000)
    l0 = dev.kernel_launches
    got = _sample(st, u2)
    used = dev.kernel_launches - l0
    amp = st.download()
    assert np.array_equal(got, O.sample(amp, n, u2))
    # the same draws on the same state once more, with the probabilities gathered
    # from the amplitudes (a Z twice leaves the state and makes them stale)
    for _ in range(2):
        L.check(L.lib.qse_apply_z(st.handle, 0))
    l1 = dev.kernel_launches
    again = _sample(st, u2)
    gathered = dev.kernel_launches - l1
    assert np.array_equal(again, got)
    assert used <= gathered, (used, gathered)


def test_unread_side_output_turns_it_off_and_samples_stay_exact(dev):
    n = 18
    st = StateVector(n, dev)
    rng = np.random.default_rng(5)
    _execute(st, _circuit("swaps", n, 3))
    _sample(st, rng.random(100))                    # on
    for seed in (4, 5, 6):                          # the second execute finds the first's output unread
        L.check(L.lib.qse_state_reset(st.handle))
        _execute(st, _circuit("swaps", n, seed))
    u = rng.random(5000)
    assert np.array_equal(_sample(st, u), O.sample(st.download(), n, u))
    idx = C.c_uint64()
    L.check(L.lib.qse_measure(st.handle, 0.25, C.byref(idx)))   # collapses: the probabilities change
    assert np.array_equal(_sample(st, u), np.full(len(u), idx.value, dtype=np.uint64))
