"""The five benchmark configurations at their stated sizes against the oracle.

  config 1  16 qubits, 20 layers of RX/RY/RZ + CNOT ladders (1260 gates):
            amplitudes <= 1e-12, then sample(4096) on a seeded uniform
            stream, bit-exact against the oracle's sampler on the device state
            and on the oracle's own state (where a target is not within
            rounding of a cumulative value);
  config 2  30 qubits, H + RZ + QFT (540 gates, 16 GiB): the state is
            downloaded and the oracle's sampler (StateVector.cpp:77-116 with
            the draws injected) runs on it for 1e6 seeded uniforms; the device
            sampler must give the same indices, bit for bit.  Then measure()
            with one draw, on the device and by the oracle on the downloaded
            state.  The number of draws whose target lies within 4 ulps of a
            cumulative boundary is reported;
  config 4  QAOA Max-Cut, random 3-regular graph on 24 nodes, p = 8 (16
            parameters, 1080 gates): value and gradient of qse_adjoint against
            the oracle's adjoint (itself checked against parameter shift at
            smaller sizes) to 1e-10, and against central finite differences
            (h = 1e-6, tolerance 1e-7) on four parameters;
  config 5  the 512-circuit batch (widths 10..22): the eight widest circuits
            (20 to 22 qubits) against the oracle's adjoint to 1e-10.
The oracle's element-wise loops and its sums run on every host core
(OpenMP, results independent of the thread count).
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle_ffi as O
from quantumsimevo_b200 import _lib as L
from quantumsimevo_b200 import workloads as W
from quantumsimevo_b200.circuit import Circuit, Device, StateVector

pytestmark = pytest.mark.gpu
TOL_AMP = 1e-12
TOL_GRAD = 1e-10


@pytest.fixture(scope="module")
def dev():
    return Device.default()


def _host_available_bytes():
    avail = None
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    avail = int(line.split()[1]) * 1024
    except OSError:
        pass
    for path in ("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory/memory.limit_in_bytes"):
        try:
            with open(path) as f:
                lim = f.read().strip()
            if lim != "max":
                used = 0
                for upath in ("/sys/fs/cgroup/memory.current", "/sys/fs/cgroup/memory/memory.usage_in_bytes"):
                    if os.path.exists(upath):
                        with open(upath) as g:
                            used = int(g.read().strip())
                        break
                cg = int(lim) - used
                avail = cg if avail is None else min(avail, cg)
        except (OSError, ValueError):
            pass
    return avail


def _free_device_bytes():
    import torch
    return torch.cuda.mem_get_info()[0]


# ---------------------------------------------------------------- config 1
def test_config1_16q_amplitudes_and_sample_4096(dev):
    n = 16
    ops = W.layered_rotations(n, 20, seed=1)
    assert len(ops) == 1260
    c = Circuit(n, device=dev, seed=1)
    c.add_ops(ops)
    c.execute()
    got_state = c.get_state_vector()
    want_state = O.run(n, ops)
    assert np.max(np.abs(got_state - want_state)) <= TOL_AMP
    u = W.SplitMix64(4096).uniforms(4096)
    got = c.sample(len(u), uniforms=u)
    # the sampler itself: bit-exact on the state it samples
    assert np.array_equal(got, O.sample(got_state, n, u))
    # end to end against the oracle's own state: equal except where a target is within
    # rounding of a cumulative value (none expected; any would be listed here)
    want = O.sample(want_state, n, u)
    cum = O.cdf(want_state, n)
    for i in np.nonzero(got != want)[0]:
        assert np.min(np.abs(cum - u[i] * cum[-1])) < 1e-12


# ---------------------------------------------------------------- config 2
def test_config2_30q_sample_1e6_and_measure_vs_oracle(dev, record_property):
    n = 30
    need_host = (16 + 8 + 2) << 30   # downloaded state + the oracle's cumulative array + slack
    avail = _host_available_bytes()
    if avail is not None and avail < need_host:
        pytest.skip(f"needs {need_host >> 30} GiB of host memory, {avail >> 30} GiB available")
    if _free_device_bytes() < (20 << 30):
        pytest.skip("needs 20 GiB of free device memory")
    ops = W.hrz_qft(n, seed=2)
    assert len(ops) == 540
    st = StateVector(n, dev)
    stats = L.QseExecStats()
    L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, None, None, 0, C.byref(stats)))
    assert stats.passes == 3
    host = st.download()            # logical order, 16 GiB
    assert host.dtype == np.complex128 and host.size == 1 << n

    u = np.random.default_rng(1_000_000).random(1_000_000)
    got = np.empty(len(u), dtype=np.uint64)
    L.check(L.lib.qse_sample(st.handle, u.ctypes.data_as(L._pd), len(u), 0, got.ctypes.data_as(L._pu64)))
    want, near = O.sample_margin(host, n, u, 4.0)
    mismatches = int(np.count_nonzero(got != want))
    record_property("draws_within_4_ulps_of_a_boundary", near)
    record_property("sample_mismatches", mismatches)
    print(f"\nconfig 2: 1e6 draws, {near} within 4 ulps of a cumulative boundary, {mismatches} mismatches")
    assert mismatches == 0, f"{mismatches} of {len(u)} outcomes differ ({near} draws near a boundary)"

    # measure(): one draw on the device state and on the downloaded copy (the oracle collapses it in place)
    um = 0.7236067977499789
    idx = C.c_uint64()
    L.check(L.lib.qse_measure(st.handle, um, C.byref(idx)))
    want_idx = O.measure_in_place(host, n, um)
    assert int(idx.value) == want_idx
    assert host[want_idx] == 1.0
    del host
    # the device state is the collapsed basis state too
    amp = np.empty(2, dtype=np.float64)
    L.check(L.lib.qse_state_download_range(st.handle, want_idx, 1, amp.ctypes.data_as(C.c_void_p)))
    assert amp[0] == 1.0 and amp[1] == 0.0


# ---------------------------------------------------------------- config 4
def _adjoint_gpu(dev, n, ops, params, obs):
    st = StateVector(n, dev)
    p = np.ascontiguousarray(params, dtype=np.float64)
    g = np.zeros(p.size)
    v = C.c_double()
    L.check(L.lib.qse_adjoint(st.handle, L.dptr(ops), len(ops), p.ctypes.data_as(L._pd), p.size, C.byref(obs),
                              C.byref(v), g.ctypes.data_as(L._pd)))
    return v.value, g, st


def _expectation_gpu(st, ops, params, obs):
    p = np.ascontiguousarray(params, dtype=np.float64)
    L.check(L.lib.qse_state_reset(st.handle))
    L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), p.ctypes.data_as(L._pd), p.size, None, None, 0,
                              None))
    v = C.c_double()
    L.check(L.lib.qse_expectation(st.handle, C.byref(obs), C.byref(v)))
    return v.value


def test_config4_qaoa_24q_p8_adjoint_vs_oracle_and_fd(dev):
    n, p = 24, 8
    ops, params, edges, obs_t = W.qaoa_maxcut(n, p, seed=4)
    assert len(edges) == 36 and params.size == 16 and len(ops) == 1080
    obs, keep = L.observable(*obs_t)
    v, g, st = _adjoint_gpu(dev, n, ops, params, obs)
    vw, gw = O.adjoint(n, ops, params, obs)
    assert abs(v - vw) <= TOL_GRAD, (v, vw)
    assert np.max(np.abs(g - gw)) <= TOL_GRAD, np.max(np.abs(g - gw))
    h = 1e-6
    for k in (0, 5, 8, 15):
        pp, pm = params.copy(), params.copy()
        pp[k] += h
        pm[k] -= h
        fd = (_expectation_gpu(st, ops, pp, obs) - _expectation_gpu(st, ops, pm, obs)) / (2 * h)
        assert abs(fd - g[k]) <= 1e-7, (k, fd, g[k])


# ---------------------------------------------------------------- config 5
def test_config5_widest_batch_circuits_vs_oracle(dev):
    from quantumsimevo_b200.batch import Batch
    hb = W.hea_batch(512, 10, 22, 4, 12, seed=5)
    circs = [(w, ops, len(pr), obs) for (w, ops, pr, obs) in hb]
    params = np.concatenate([pr for (_, _, pr, _) in hb])
    off = np.concatenate([[0], np.cumsum([c[2] for c in circs])])
    widest = sorted(range(len(circs)), key=lambda i: (-circs[i][0], i))[:8]
    assert min(circs[i][0] for i in widest) >= 20
    b = Batch(circs, dev)
    v, g = b.run(params)
    for i in widest:
        obs, keep = L.observable(*circs[i][3])
        vw, gw = O.adjoint(circs[i][0], circs[i][1], params[off[i]:off[i + 1]], obs)
        assert abs(v[i] - vw) <= TOL_GRAD, (i, v[i], vw)
        assert np.max(np.abs(g[off[i]:off[i + 1]] - gw)) <= TOL_GRAD, (i, np.max(np.abs(g[off[i]:off[i + 1]] - gw)))


# ---------------------------------------------------------------- adjoint at 30 qubits
def test_adjoint_30q_on_one_gpu(dev, record_property):
    """The adjoint sweep keeps two 16 GiB states (psi and lambda) at 30 qubits:
    Max-Cut QAOA on a random 3-regular graph with 30 nodes, p = 1.  The value
    must equal qse_expectation after a plain execute, and both gradient entries
    the parameter-shift rule on the same engine (2 executes per parameterised
    occurrence, 330 executes)."""
    import math
    if _free_device_bytes() < (40 << 30):
        pytest.skip("needs 40 GiB of free device memory")
    n = 30
    ops, params, edges, obs_t = W.qaoa_maxcut(n, 1, seed=30)
    assert len(edges) == 45
    obs, keep = L.observable(*obs_t)
    v, g, st = _adjoint_gpu(dev, n, ops, params, obs)
    e = _expectation_gpu(st, ops, params, obs)
    assert abs(v - e) <= 1e-10 * max(1.0, abs(e)), (v, e)
    occ = [i for i in range(len(ops)) if int(ops[i]["param"]) >= 0]
    bound = ops.copy()
    for i in occ:
        bound[i]["theta"] = ops[i]["theta"] + ops[i]["coeff"] * params[int(ops[i]["param"])]
        bound[i]["param"] = -1
        bound[i]["coeff"] = 1.0
    g_ps = np.zeros(params.size)
    work = bound.copy()
    for i in occ:
        th = bound[i]["theta"]
        work[i]["theta"] = th + math.pi / 2
        fp = _expectation_gpu(st, work, np.zeros(0), obs)
        work[i]["theta"] = th - math.pi / 2
        fm = _expectation_gpu(st, work, np.zeros(0), obs)
        work[i]["theta"] = th
        g_ps[int(ops[i]["param"])] += ops[i]["coeff"] * (fp - fm) / 2
    diff = float(np.max(np.abs(g - g_ps)))
    record_property("adjoint_30q_max_abs_diff_vs_param_shift", diff)
    print(f"\nadjoint 30q: value {v:.15f}, grad {g}, max |adjoint - parameter shift| = {diff:.3e}")
    assert diff <= 1e-9, (g, g_ps)
