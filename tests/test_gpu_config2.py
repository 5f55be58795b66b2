"""The 30-qubit bench circuit (H on all qubits, RZ, full QFT: 540 gates, 16 GiB of
complex128 amplitudes) at full size.  The FP64 oracle cannot hold this state, so
parity is checked through properties that do not depend on size:
  - unit norm: the tree-reduced sum of |amplitude|^2 on the device to 1e-12,
    and the reference's sequentially rounded total (qse_total_probability)
    within the bound of recursive summation, (N-1) u = 2^30 * 2^-53;
  - sorted uniforms give non-decreasing outcome indices (the exact cumulative
    array is monotone and the search is a lower bound), over 1e5 shots;
  - the inverse circuit returns the state to |0..0> (|amplitude 0| = 1 within
    1e-9), which holds only if every gate, the fusion plan, the deferred pass
    constants and the SWAP relabelling were applied as the reference defines.
The same circuit at 20 qubits is compared amplitude by amplitude with the oracle
in test_gpu_core.py (test_qft_20q)."""
import ctypes as C

import numpy as np
import pytest

from quantumsimevo_b200 import _lib as L
from quantumsimevo_b200 import workloads as W
from quantumsimevo_b200.circuit import Device, StateVector
from test_gpu_config3 import amp0, execute, inverse_ops

pytestmark = pytest.mark.gpu


def test_hrz_qft_30q_norm_sampler_and_round_trip():
    dev = Device.default()
    free, _ = __import__("torch").cuda.mem_get_info()
    n = 30
    if free < (24 << 30):
        pytest.skip("needs 16 GiB of free device memory")
    ops = W.hrz_qft(n, seed=2)
    assert len(ops) == 540
    st = StateVector(n, dev)
    stats = execute(st, ops)
    assert stats.passes == 3
    import torch
    from quantumsimevo_b200.sharded import _DeviceArray
    dev.synchronize()
    p = C.c_void_p()
    L.check(L.lib.qse_state_device_ptr(st.handle, C.byref(p)))
    view = torch.as_tensor(_DeviceArray(p.value, 1 << n), device=f"cuda:{dev.index}")
    assert abs(float(torch.linalg.vector_norm(view)) ** 2 - 1.0) <= 1e-12
    total = C.c_double()
    L.check(L.lib.qse_total_probability(st.handle, C.byref(total)))
    assert abs(total.value - 1.0) <= 2.0 ** 30 * 2.0 ** -53
    u = np.sort(np.random.default_rng(30).random(100_000))
    out = np.empty(len(u), dtype=np.uint64)
    L.check(L.lib.qse_sample(st.handle, u.ctypes.data_as(L._pd), len(u), 0, out.ctypes.data_as(L._pu64)))
    assert np.all(np.diff(out.astype(np.int64)) >= 0)
    assert int(out[-1]) < (1 << n)
    execute(st, inverse_ops(ops))
    assert abs(abs(amp0(st)) - 1.0) <= 1e-9
