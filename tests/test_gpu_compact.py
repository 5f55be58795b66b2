"""Executes whose leading passes run on a compact state.

A circuit started from a basis state reaches its qubits progressively; while
the qubits touched so far number at most 22, the engine runs those passes on
a state of only the touched qubits and the first pass over the full state
reads its input from it (engine.cu compact_prefix, jit.cpp compact input).
Checked against the oracle on 24-qubit states:
  - gates in three waves (12 qubits, 22 qubits, all 24) from |0..0>;
  - the same from a basis state left by measure() (nonzero bits on the
    untouched qubits, relabelled qubits from earlier SWAPs);
  - a circuit that never leaves 22 qubits (the compact state is written out);
and the 26-qubit H+RZ+QFT against the same circuit from an uploaded |0..0>
(no compact prefix), with the full-state pass counts of both.
Product qubits (engine.cu absorb_product_qubits): qubits the prefix leaves in a
basis state whose next gates act on them alone hold a single-qubit state each,
which the first full-state pass multiplies into its input.  Checked with such
qubits on register, thread and outer bits of that pass, from |0..0> and from a
measured basis state, and with every gate after the prefix absorbed (the
product form written out).
"""
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


ONE_QUBIT = [W.H, W.X, W.Y, W.Z, W.PHASE, W.RX, W.RY, W.RZ, W.GATE2X2]


def _one_qubit_layer(qubits, count, seed):
    """count random one-qubit gates (every kind) on the given qubits."""
    ops = W.random_circuit(len(qubits), count, seed, types=ONE_QUBIT)
    ops["target"] = np.asarray(qubits, dtype=np.uint32)[ops["target"]]
    return ops


def _waves(sizes, counts, seed):
    return np.concatenate([W.random_circuit(k, c, seed + i) for i, (k, c) in enumerate(zip(sizes, counts))])


def _execute(st, ops):
    stats = L.QseExecStats()
    L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, None, None, 0, C.byref(stats)))
    return stats


def _full_state_passes(dev, st, ops):
    """(passes reported, passes over the full state) of one execute: the pass
    timings list only full-state passes."""
    L.check(L.lib.qse_ctx_time_passes(dev.handle, 1))
    pl = np.zeros(64)
    cnt = C.c_size_t()
    L.check(L.lib.qse_ctx_pass_time_list(dev.handle, pl.ctypes.data_as(L._pd), pl.size, C.byref(cnt)))
    stats = _execute(st, ops)
    dev.synchronize()
    L.check(L.lib.qse_ctx_pass_time_list(dev.handle, pl.ctypes.data_as(L._pd), pl.size, C.byref(cnt)))
    L.check(L.lib.qse_ctx_time_passes(dev.handle, 0))
    return int(stats.passes), int(cnt.value)


def test_three_waves_from_zero(dev):
    n = 24
    ops = _waves([12, 22, 24], [160, 320, 120], 41)
    st = StateVector(n, dev)
    total, full = _full_state_passes(dev, st, ops)
    assert full < total, (total, full)        # some passes ran on the compact state
    assert np.max(np.abs(st.download() - O.run(n, ops))) <= TOL


def test_three_waves_from_measured_basis_state(dev):
    n = 24
    first = np.concatenate([W.random_circuit(n, 60, 7), W.to_array(W.qft_ops(n))])   # ends in SWAPs: relabelled
    st = StateVector(n, dev)
    _execute(st, first)
    # a draw whose outcome has logical qubits 22 and 23 (left untouched by the
    # waves' first two) at 1
    amp = st.download()
    cum = O.cdf(amp, n)
    j = next(x for x in range(3 << 22, 1 << n) if cum[x] > cum[x - 1])
    u = 0.5 * (cum[j - 1] + cum[j]) / cum[-1]
    idx = C.c_uint64()
    L.check(L.lib.qse_measure(st.handle, u, C.byref(idx)))
    i = int(idx.value)
    assert i == j
    ops = _waves([12, 22, 24], [160, 320, 120], 43)
    total, full = _full_state_passes(dev, st, ops)
    assert full < total, (total, full)
    start = np.zeros(1 << n, dtype=np.complex128)
    start[i] = 1.0
    assert np.max(np.abs(st.download() - O.run_on(start, n, ops))) <= TOL


def test_circuit_within_22_qubits_is_written_out(dev):
    n = 24
    ops = _waves([12, 22], [160, 400], 45)
    st = StateVector(n, dev)
    total, full = _full_state_passes(dev, st, ops)
    assert full == 0 and total >= 2, (total, full)
    assert np.max(np.abs(st.download() - O.run(n, ops))) <= TOL


def test_hrz_qft_26q_against_uploaded_start(dev):
    n = 26
    ops = W.hrz_qft(n, seed=2)
    st = StateVector(n, dev)
    total, full = _full_state_passes(dev, st, ops)
    got = st.download()
    ref = StateVector(n, dev)
    zero = np.zeros(1 << n, dtype=np.complex128)
    zero[0] = 1.0
    ref.upload(zero)                           # a written |0..0>: every pass over the full state
    total_r, full_r = _full_state_passes(dev, ref, ops)
    assert full < full_r, (total, full, total_r, full_r)
    assert np.max(np.abs(got - ref.download())) <= TOL


def test_product_qubits_after_the_prefix(dev):
    """Qubits 22..25 of 26 take one-qubit gates after two waves on 22 qubits;
    then 22..24 meet H and CNOTs (tile bits of the full pass) while 25 meets only
    phases with the others (an outer bit there)."""
    n = 26
    tail = np.concatenate([W.random_circuit(n - 1, 80, 71),
                           W.to_array([W._op(W.CPHASE, 25, k, theta=0.3 * (k + 1)) for k in range(0, 25, 3)])])
    ops = np.concatenate([_waves([12, 22], [160, 320], 61), _one_qubit_layer([22, 23, 24, 25], 40, 62), tail])
    st = StateVector(n, dev)
    total, full = _full_state_passes(dev, st, ops)
    assert full < total, (total, full)
    assert np.max(np.abs(st.download() - O.run(n, ops))) <= TOL


def test_product_qubits_from_measured_basis_state(dev):
    n = 24
    st = StateVector(n, dev)
    _execute(st, W.to_array([W._op(W.X, 22), W._op(W.X, 23), W._op(W.H, 5)]))
    idx = C.c_uint64()
    L.check(L.lib.qse_measure(st.handle, 0.75, C.byref(idx)))   # |0..0> + qubits 22, 23 (and maybe 5) set
    i = int(idx.value)
    assert (i >> 22) & 3 == 3
    ops = np.concatenate([_waves([12, 22], [160, 320], 63), _one_qubit_layer([22, 23], 12, 64),
                          W.random_circuit(n, 60, 65)])
    total, full = _full_state_passes(dev, st, ops)
    assert full < total, (total, full)
    start = np.zeros(1 << n, dtype=np.complex128)
    start[i] = 1.0
    assert np.max(np.abs(st.download() - O.run_on(start, n, ops))) <= TOL


def test_every_gate_after_the_prefix_absorbed(dev):
    """Nothing is left for a full-state pass: the product form is written out."""
    n = 24
    # (waves whose passes finish before any gate on 22, 23 needs a tile: every
    # gate after the prefix is one of the layer's)
    ops = np.concatenate([_waves([12, 22], [160, 320], 74), _one_qubit_layer([22, 23], 10, 67)])
    st = StateVector(n, dev)
    total, full = _full_state_passes(dev, st, ops)
    assert full == 0 and total >= 2, (total, full)
    assert np.max(np.abs(st.download() - O.run(n, ops))) <= TOL
