"""32-qubit random layers with Pauli noise (64 GiB of complex128 amplitudes):
40 layers of one random single-qubit gate per qubit, 16 disjoint random
CNOT / CPHASE / SWAP pairs and one 3-control MCPHASE, every gate of the
reference's error-rate map (Noise.cpp:10-18) at p = 1e-3, Philox draws.

The FP64 oracle cannot hold this state, so parity is checked through
properties that do not depend on size:
  - the noise decisions (per-qubit bit- and phase-flip counts) are bit-exact
    against the oracle's Noise.cpp restatement, which needs only the gate list
    and the draws;
  - the state keeps unit norm (the reference's sequential sum, to 1e-10);
  - undoing the Pauli frame and then applying the inverse circuit returns the
    state to |0..0> (|amplitude 0| = 1 within 1e-9), which holds only if every
    one of the 1960 gates, the fusion plan and the qubit relabelling by SWAP
    were applied exactly as the reference defines them.
Smaller instances of the same generator are compared amplitude by amplitude
with the oracle in test_gpu_core.py (random circuits, noise)."""
import ctypes as C

import numpy as np
import pytest

import oracle_ffi as O
from quantumsimevo_b200 import _lib as L
from quantumsimevo_b200 import workloads as W
from quantumsimevo_b200.circuit import Device, Noise, StateVector

pytestmark = pytest.mark.gpu


def inverse_ops(ops):
    inv = ops[::-1].copy()
    for i in range(len(inv)):
        if int(inv[i]["type"]) in (L.RX, L.RY, L.RZ, L.PHASE, L.CPHASE, L.MCPHASE):
            inv[i]["theta"] = -inv[i]["theta"]
    return np.ascontiguousarray(inv)


def execute(st, ops, noise=None):
    stats = L.QseExecStats()
    L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, noise.handle if noise else None, None, 0,
                              C.byref(stats)))
    return stats


def amp0(st):
    out = np.zeros(2, dtype=np.float64)
    L.check(L.lib.qse_state_download_range(st.handle, 0, 1, out.ctypes.data_as(C.c_void_p)))
    return complex(out[0], out[1])


def test_random_layers_32q_with_noise():
    dev = Device.default()
    free, _ = __import__("torch").cuda.mem_get_info()
    n = 32
    if free < (70 << 30):
        pytest.skip("needs 64 GiB of free device memory")
    ops = W.random_layers(n, 40, seed=3)
    assert len(ops) == 1960
    rates = W.noise_rates(1e-3)
    cfg = L.default_noise_config(True, L.RNG_PHILOX, 2024, 1.0, rates)
    want_bits, want_phases = O.noise_decisions(n, ops, cfg)

    st = StateVector(n, dev)
    nz = Noise(n, 2024, 1.0, L.RNG_PHILOX, rates=rates, device=dev)
    stats = execute(st, ops, nz)
    assert stats.gates == len(ops)
    bits, phases = nz.counts()
    assert bits == want_bits and phases == want_phases
    assert sum(bits) + sum(phases) > 0

    total = C.c_double()
    L.check(L.lib.qse_total_probability(st.handle, C.byref(total)))
    assert abs(total.value - 1.0) <= 1e-10

    # undo the end-of-execute Pauli frame (X then Z per qubit), then the circuit
    for q in range(n):
        if phases[q] % 2:
            L.check(L.lib.qse_apply_z(st.handle, q))
        if bits[q] % 2:
            L.check(L.lib.qse_apply_x(st.handle, q))
    execute(st, inverse_ops(ops))
    a = amp0(st)
    assert abs(abs(a) - 1.0) <= 1e-9, a
