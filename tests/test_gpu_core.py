"""GPU parity: the CUDA path through the C ABI against the oracle.

Amplitudes: max abs error <= 1e-12 (the reference's KAT tolerance,
QSETests.cpp:40).  Sample / measure outcome indices and noise decisions:
bit-exact for the same uniform draws.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_ffi as O
from quantumsimevo_b200 import _lib as L
from quantumsimevo_b200 import workloads as W
from quantumsimevo_b200.circuit import Circuit, Device, Noise, StateVector

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def dev():
    return Device.default()


def run_gpu(dev, n, ops, fusion=True, k=0, max_gates=0, params=None):
    dev.set_fusion(fusion, k, max_gates)
    st = StateVector(n, dev)
    ops = np.ascontiguousarray(ops)
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
    stats = L.QseExecStats()
    L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), p.ctypes.data_as(L._pd) if p is not None else None,
                              0 if p is None else p.size, None, None, 0, C.byref(stats)))
    out = st.download()
    dev.set_fusion(True, 12, 0)
    return out, stats


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 10, 13])
def test_plain_kernels_every_gate_every_qubit(dev, n):
    ops = W.random_circuit(n, 40 * n, 100 + n)
    got, stats = run_gpu(dev, n, ops, fusion=False)
    assert np.max(np.abs(got - O.run(n, ops))) <= TOL


@pytest.mark.parametrize("n,k", [(4, 4), (6, 5), (9, 9), (10, 8), (12, 12), (13, 10), (14, 12), (16, 11), (18, 12)])
def test_fused_random_circuits(dev, n, k):
    for rep in range(3):
        ops = W.random_circuit(n, 25 * n, 3000 + 7 * n + rep)
        got, stats = run_gpu(dev, n, ops, fusion=True, k=k)
        err = np.max(np.abs(got - O.run(n, ops)))
        assert err <= TOL, (rep, err, stats.passes)


@pytest.mark.parametrize("n,k", [(6, 5), (12, 12), (14, 10)])
def test_interpreter_kernel_without_jit(dev, n, k):
    """The generic pass kernel (interpreter of the planned programs) that runs
    when the NVRTC-specialised kernels are switched off; forward and adjoint."""
    L.check(L.lib.qse_ctx_set_jit(dev.handle, 0))
    try:
        ops = W.random_circuit(n, 25 * n, 5000 + n)
        got, _ = run_gpu(dev, n, ops, fusion=True, k=k)
        assert np.max(np.abs(got - O.run(n, ops))) <= TOL
        qops, params, _, obs_t = W.qaoa_maxcut(n, 2, seed=50 + n)
        v, g = _adjoint(dev, n, qops, params, obs_t)
        obs, keep = L.observable(*obs_t)
        vw, gw = O.adjoint(n, qops, params, obs)
        assert abs(v - vw) <= 1e-10
        assert np.max(np.abs(g - gw)) <= 1e-10
    finally:
        L.check(L.lib.qse_ctx_set_jit(dev.handle, 1))


def test_fused_gate_cap_and_tiles(dev):
    n = 15
    ops = W.random_circuit(n, 400, 42)
    want = O.run(n, ops)
    for k, cap in [(9, 3), (10, 0), (11, 17), (12, 1)]:
        got, _ = run_gpu(dev, n, ops, k=k, max_gates=cap)
        assert np.max(np.abs(got - want)) <= TOL


def test_layered_rotations_16q_full(dev):
    ops = W.layered_rotations(16, 20, seed=1)
    got, stats = run_gpu(dev, 16, ops)
    assert np.max(np.abs(got - O.run(16, ops))) <= TOL
    assert stats.passes < 20


def test_qft_20q(dev):
    ops = W.hrz_qft(20, seed=2)
    got, stats = run_gpu(dev, 20, ops)
    assert np.max(np.abs(got - O.run(20, ops))) <= TOL
    assert stats.passes <= 4


def test_reset_then_every_reader_sees_zero_state(dev):
    """Reset records |0..0> without writing the array; the next fused execute
    generates it in its first pass and every other reader writes it first."""
    n = 13
    ops = W.random_circuit(n, 120, 17)
    want = O.run(n, ops)
    zero = np.zeros(1 << n, dtype=np.complex128)
    zero[0] = 1.0
    st = StateVector(n, dev)

    def dirty():
        L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, None, None, 0, None))
        L.check(L.lib.qse_state_reset(st.handle))

    dirty()
    assert np.array_equal(st.download(), zero)
    dirty()
    L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, None, None, 0, None))
    assert np.max(np.abs(st.download() - want)) <= TOL
    dirty()
    L.check(L.lib.qse_apply_h(st.handle, 0))
    h = zero.copy()
    h[0] = h[1] = 1 / np.sqrt(2)
    assert np.max(np.abs(st.download() - h)) <= TOL
    dirty()
    out = np.zeros(8, dtype=np.uint64)
    L.check(L.lib.qse_sample(st.handle, np.linspace(0.01, 0.99, 8).ctypes.data_as(L._pd), 8, 0,
                             out.ctypes.data_as(L._pu64)))
    assert np.all(out == 0)
    dirty()
    obs, keep = L.observable([1, 2], [1.0, 0.5], 0.25)
    v = C.c_double()
    L.check(L.lib.qse_expectation(st.handle, C.byref(obs), C.byref(v)))
    assert abs(v.value - 1.75) <= TOL
    dirty()
    dev.set_fusion(False)
    L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, None, None, 0, None))
    dev.set_fusion(True, 12, 0)
    assert np.max(np.abs(st.download() - want)) <= TOL
    dirty()
    swaps = W.to_array([(L.SWAP, 0, 5, -1, 0, 0.0, 1.0, (0.0,) * 8)] * 3)
    L.check(L.lib.qse_execute(st.handle, L.dptr(swaps), len(swaps), None, 0, None, None, 0, None))
    assert np.array_equal(st.download(), zero)


def test_measure_then_every_reader_sees_the_basis_state(dev):
    """measure() records the outcome's basis state without writing the array:
    the next fused execute generates it in its first pass (kernel shared with
    reset, the index in its parameter block), every other reader writes it
    first, and a reset discards it.  Relabelled qubits (swaps before the measure)
    included; states of 13 and 23 qubits (one tile / many tiles per pass)."""
    for n in (13, 23):
        pre = np.concatenate([W.random_circuit(n, 60, 31 + n), W.to_array(W.qft_ops(n))])
        ops = W.random_circuit(n, 80, 41 + n)
        st = StateVector(n, dev)

        def measured(u):
            L.check(L.lib.qse_state_reset(st.handle))
            L.check(L.lib.qse_execute(st.handle, L.dptr(pre), len(pre), None, 0, None, None, 0, None))
            idx = C.c_uint64()
            L.check(L.lib.qse_measure(st.handle, u, C.byref(idx)))
            basis = np.zeros(1 << n, dtype=np.complex128)
            basis[int(idx.value)] = 1.0
            return basis

        for u in (0.1, 0.77):
            basis = measured(u)
            assert np.array_equal(st.download(), basis)
            basis = measured(u)
            L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, None, None, 0, None))
            assert np.max(np.abs(st.download() - O.run_on(basis, n, ops))) <= TOL
            basis = measured(u)
            dev.set_fusion(False)
            L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, None, None, 0, None))
            dev.set_fusion(True, 12, 0)
            assert np.max(np.abs(st.download() - O.run_on(basis, n, ops))) <= TOL
            basis = measured(u)
            uu = np.linspace(0.01, 0.99, 8)
            out = np.zeros(8, dtype=np.uint64)
            L.check(L.lib.qse_sample(st.handle, uu.ctypes.data_as(L._pd), 8, 0, out.ctypes.data_as(L._pu64)))
            assert np.all(out == np.flatnonzero(basis)[0])
            measured(u)
            L.check(L.lib.qse_state_reset(st.handle))
            L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, None, None, 0, None))
            assert np.max(np.abs(st.download() - O.run(n, ops))) <= TOL


def test_execute_twice_and_swap_relabel(dev):
    # Circuit::execute does not clear its queue: a second execute applies it again
    n = 11
    ops = W.random_circuit(n, 120, 5)
    c = Circuit(n, device=dev, seed=3)
    c.add_ops(ops)
    c.execute()
    c.execute()
    want = O.run_on(O.run(n, ops), n, ops)
    assert np.max(np.abs(c.get_state_vector() - want)) <= TOL


def test_per_gate_api_after_fused_relabel(dev):
    # a fused execute leaves a qubit relabelling; per-gate calls must honour it
    n = 10
    ops = W.to_array([(L.SWAP, 0, 9, -1, 0, 0.0, 1.0, (0.0,) * 8), (L.H, 0, 0, -1, 0, 0.0, 1.0, (0.0,) * 8),
                      (L.SWAP, 1, 5, -1, 0, 0.0, 1.0, (0.0,) * 8)])
    st = StateVector(n, dev)
    L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, None, None, 0, None))
    L.check(L.lib.qse_apply_rx(st.handle, 0, 0.3))
    L.check(L.lib.qse_apply_cnot(st.handle, 0, 5))
    more = W.to_array([(L.RX, 0, 0, -1, 0, 0.3, 1.0, (0.0,) * 8), (L.CNOT, 5, 0, -1, 0, 0.0, 1.0, (0.0,) * 8)])
    want = O.run(n, np.concatenate([ops, more]))
    assert np.max(np.abs(st.download() - want)) <= TOL
    L.check(L.lib.qse_state_canonicalize(st.handle))
    assert st.qubit_map() == list(range(n))
    assert np.max(np.abs(st.download() - want)) <= TOL


def test_errors_are_status_codes(dev):
    st = StateVector(4, dev)
    assert L.lib.qse_apply_h(st.handle, 4) == 2
    ops = L.as_ops([L.make_op(L.CNOT, 1, 9)])
    assert L.lib.qse_execute(st.handle, L.dptr(ops), 1, None, 0, None, None, 0, None) == 2
    h = C.c_void_p()
    assert L.lib.qse_state_create(dev.handle, 80, C.byref(h)) == 5
    # the context is still usable
    L.check(L.lib.qse_apply_h(st.handle, 3))


# ---------------------------------------------------------------- sampling
def boundary_uniforms(st, n, count, seed):
    """Uniforms that put targets exactly on and next to cumulative values."""
    cum = O.cdf(st, n)
    total = cum[-1]
    rng = np.random.default_rng(seed)
    picks = rng.integers(0, cum.size, count)
    u = []
    for i in picks:
        x = cum[i] / total
        for v in (x, np.nextafter(x, 0.0), np.nextafter(x, 1.0)):
            if 0.0 <= v < 1.0:
                u.append(v)
    u += list(rng.random(count))
    return np.array(u, dtype=np.float64)


def _sample_on(dev, n, amp, u):
    st = StateVector(n, dev)
    st.upload(amp)
    out = np.empty(len(u), dtype=np.uint64)
    L.check(L.lib.qse_sample(st.handle, u.ctypes.data_as(L._pd), len(u), 0, out.ctypes.data_as(L._pu64)))
    return out


@pytest.mark.parametrize("n", [1, 3, 8, 11, 12, 13, 16, 20])
def test_sample_bit_exact(dev, n):
    # the sampler alone: the oracle's state uploaded, draws on and beside every kind of boundary
    ops = W.random_circuit(n, 20 * n, 600 + n)
    st = O.run(n, ops)
    u = boundary_uniforms(st, n, 300, n)
    assert np.array_equal(_sample_on(dev, n, st, u), O.sample(st, n, u))


@pytest.mark.parametrize("spread", [0.0, 40.0])
def test_sample_bit_exact_many_blocks(dev, spread):
    # 2048 blocks of 4096: every persistent CTA of the CDF write takes several
    # blocks and the chain several 1024-block chunks; spread > 0 puts the
    # magnitudes over many binades so the slow paths run inside those loops
    n = 23
    rng = np.random.default_rng(23 + int(spread))
    amp = (rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)) * np.exp(-rng.uniform(0, spread, 1 << n))
    amp /= np.linalg.norm(amp)
    u = boundary_uniforms(amp, n, 400, 4)
    assert np.array_equal(_sample_on(dev, n, amp, u), O.sample(amp, n, u))


def test_sample_spans_with_zero_regions(dev):
    """The chain composes spans of 4096 blocks: 25 qubits = 8192 blocks, with
    the first 3/8 of the amplitudes zero (the running sum is 0: the subnormal
    grid's fast path), a zero gap in the middle and magnitudes over many
    binades elsewhere (spans that stop at a block leaving its binade and
    restart after it), against the oracle's sampler.  The statistics show the
    zero blocks composed in spans, not folded one by one."""
    n = 25
    rng = np.random.default_rng(2525)
    size = 1 << n
    mag = np.exp(-rng.uniform(0, 30, size))
    mag[: 3 * size // 8] = 0.0
    mag[size // 2: size // 2 + size // 16] = 0.0
    amp = mag * np.exp(1j * rng.uniform(0, 2 * np.pi, size))
    amp /= np.linalg.norm(amp)
    st = StateVector(n, dev)
    st.upload(amp)
    u = boundary_uniforms(amp, n, 300, 25)
    out = np.empty(len(u), dtype=np.uint64)
    L.check(L.lib.qse_sample(st.handle, u.ctypes.data_as(L._pd), len(u), 0, out.ctypes.data_as(L._pu64)))
    assert np.array_equal(out, O.sample(amp, n, u))
    stats = (C.c_uint32 * 4)()
    L.check(L.lib.qse_sampler_stats(st.handle, stats))
    spans, single, exact, nb = list(stats)
    assert nb == size // 4096
    assert exact < 64 and single < 64, list(stats)


@pytest.mark.parametrize("n", [5, 14, 18])
def test_sample_after_execute(dev, n):
    # end to end: outcomes equal the oracle's sampler on the device state; against the
    # oracle's own state they may differ only where a target is within rounding of a CDF value
    ops = W.random_circuit(n, 20 * n, 650 + n)
    c = Circuit(n, device=dev, seed=9)
    c.add_ops(ops)
    c.execute()
    u = np.random.default_rng(n).random(5000)
    got = c.sample(len(u), uniforms=u)
    dev_state = c.get_state_vector()
    assert np.array_equal(got, O.sample(dev_state, n, u))
    st = O.run(n, ops)
    want = O.sample(st, n, u)
    cum = O.cdf(st, n)
    for i in np.nonzero(got != want)[0]:
        t = u[i] * cum[-1]
        assert np.min(np.abs(cum - t)) < 1e-12

def test_sample_bucketed_shot_patterns(dev):
    """The shots are bucketed by block and each block with shots rebuilds its
    exact cumulative values in shared memory: one shot, a handful, tens of
    thousands in one block (identical draws), draws at 0 and just below 1, and
    every block touched -- against the oracle's sampler on the same state."""
    n = 21
    ops = W.random_circuit(n, 10 * n, 777)
    st = StateVector(n, dev)
    L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, None, None, 0, None))
    amp = st.download()
    cases = [np.array([0.5]), np.array([0.0, 0.999999, 0.25, 0.75, 0.5]),
             np.full(40000, 0.3141592653589793), np.array([0.0, 1.0 - 2.0 ** -53]),
             np.random.default_rng(21).random(300000)]
    for u in cases:
        out = np.empty(len(u), dtype=np.uint64)
        L.check(L.lib.qse_sample(st.handle, u.ctypes.data_as(L._pd), len(u), 0, out.ctypes.data_as(L._pu64)))
        assert np.array_equal(out, O.sample(amp, n, u)), len(u)


def test_sample_exact_cdf_many_binades(dev):
    # amplitudes spread over many binades so the running sum crosses many
    # binade boundaries inside blocks (the exact scan's slow path)
    n = 16
    rng = np.random.default_rng(5)
    mag = np.exp(rng.uniform(-60, 0, 1 << n))
    amp = mag * np.exp(1j * rng.uniform(0, 2 * np.pi, 1 << n))
    amp[:100] = 0.0
    amp[5000:5003] = 1e-160
    st = StateVector(n, dev)
    st.upload(amp)
    u = boundary_uniforms(amp, n, 500, 1)
    out = np.empty(len(u), dtype=np.uint64)
    L.check(L.lib.qse_sample(st.handle, u.ctypes.data_as(L._pd), len(u), 0, out.ctypes.data_as(L._pu64)))
    assert np.array_equal(out, O.sample(amp, n, u))
    t = C.c_double()
    L.check(L.lib.qse_total_probability(st.handle, C.byref(t)))
    assert t.value == O.cdf(amp, n)[-1]


def test_sample_ties_to_even(dev):
    # probabilities that are exact multiples of half-ulps exercise the tie rule
    n = 14
    p = np.full(1 << n, 2.0 ** -14)
    p[1::3] = 2.0 ** -14 + 2.0 ** -67
    amp = np.sqrt(p).astype(np.complex128)
    st = StateVector(n, dev)
    st.upload(amp)
    u = boundary_uniforms(amp, n, 400, 2)
    out = np.empty(len(u), dtype=np.uint64)
    L.check(L.lib.qse_sample(st.handle, u.ctypes.data_as(L._pd), len(u), 0, out.ctypes.data_as(L._pu64)))
    assert np.array_equal(out, O.sample(amp, n, u))


def test_measure_collapses(dev):
    n = 12
    ops = W.random_circuit(n, 200, 8)
    c = Circuit(n, device=dev, seed=1)
    c.add_ops(ops)
    c.execute()
    st = c.get_state_vector()
    u = 0.6180339887
    idx_want, st_want = O.measure(st, n, u)
    assert c.measure(u) == idx_want
    assert np.array_equal(c.get_state_vector(), st_want)


def test_sample_after_relabel_is_logical(dev):
    n = 13
    ops = np.concatenate([W.random_circuit(n, 100, 12), W.to_array(W.qft_ops(n))])
    c = Circuit(n, device=dev, seed=2)
    c.add_ops(ops)
    c.execute()
    st = c.get_state_vector()   # logical order after the swap relabelling
    assert np.max(np.abs(st - O.run(n, ops))) <= TOL
    u = boundary_uniforms(st, n, 200, 3)
    assert np.array_equal(c.sample(len(u), uniforms=u), O.sample(st, n, u))


# ---------------------------------------------------------------- noise
def _noisy(dev, n, ops, rng_mode, seed=42, mult=1.0, uniforms=None, rates=None):
    nz = Noise(n, seed, mult, rng_mode, rates=rates, device=dev)
    st = StateVector(n, dev)
    u = None if uniforms is None else np.ascontiguousarray(uniforms, dtype=np.float64)
    stats = L.QseExecStats()
    L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, nz.handle,
                              u.ctypes.data_as(L._pd) if u is not None else None, 0 if u is None else u.size,
                              C.byref(stats)))
    return st.download(), nz.counts(), stats


@pytest.mark.parametrize("n", [5, 12])
def test_noise_injected_uniforms_bit_exact(dev, n):
    ops = W.random_circuit(n, 300, 70 + n)
    rates = W.noise_rates(1e-3)
    cfg = L.default_noise_config(True, L.RNG_INJECTED, 42, 50.0, rates)
    noisy = int(np.sum(np.isin(ops["type"], list(rates))))
    u = np.random.default_rng(n).random(2 * noisy)
    st_want, nz = O.execute_noisy(n, ops, cfg, uniforms=u)
    st, (bits, phases), stats = _noisy(dev, n, ops, L.RNG_INJECTED, mult=50.0, uniforms=u, rates=rates)
    assert stats.noisy_gates == noisy
    assert bits == list(nz.bit[:n]) and phases == list(nz.phase[:n])
    assert sum(bits) > 0
    assert np.max(np.abs(st - st_want)) <= TOL


def test_noise_philox_matches_oracle_philox(dev):
    n = 10
    ops = W.random_circuit(n, 500, 71)
    cfg = L.default_noise_config(True, L.RNG_PHILOX, 1234, 100.0)
    st_want, nz = O.execute_noisy(n, ops, cfg)
    st, (bits, phases), _ = _noisy(dev, n, ops, L.RNG_PHILOX, seed=1234, mult=100.0)
    assert bits == list(nz.bit[:n]) and phases == list(nz.phase[:n])
    assert np.max(np.abs(st - st_want)) <= TOL


def test_noise_mt19937_matches_reference_stream(dev):
    # QSE_RNG_MT19937 consumes mt19937(42) like Noise.cpp; counts match the oracle's restatement
    n = 8
    ops = W.random_circuit(n, 400, 72)
    cfg = L.default_noise_config(True, L.RNG_MT19937, 42, 30.0)
    st_want, nz = O.execute_noisy(n, ops, cfg)
    st, (bits, phases), _ = _noisy(dev, n, ops, L.RNG_MT19937, seed=42, mult=30.0)
    assert bits == list(nz.bit[:n]) and phases == list(nz.phase[:n])
    assert np.max(np.abs(st - st_want)) <= TOL


# ---------------------------------------------------------------- gradients
def _adjoint(dev, n, ops, params, obs_t):
    obs, keep = L.observable(*obs_t)
    st = StateVector(n, dev)
    p = np.ascontiguousarray(params, dtype=np.float64)
    g = np.zeros(p.size)
    v = C.c_double()
    L.check(L.lib.qse_adjoint(st.handle, L.dptr(ops), len(ops), p.ctypes.data_as(L._pd), p.size, C.byref(obs),
                              C.byref(v), g.ctypes.data_as(L._pd)))
    return v.value, g


@pytest.mark.parametrize("n", [6, 10, 12])
def test_adjoint_qaoa_vs_oracle(dev, n):
    ops, params, edges, obs_t = W.qaoa_maxcut(n, 3, seed=40 + n)
    v, g = _adjoint(dev, n, ops, params, obs_t)
    obs, keep = L.observable(*obs_t)
    vw, gw = O.adjoint(n, ops, params, obs)
    vs, gs = O.param_shift(n, ops, params, obs)
    assert abs(v - vw) <= 1e-10
    assert np.max(np.abs(g - gw)) <= 1e-10
    assert np.max(np.abs(g - gs)) <= 1e-10


def test_adjoint_every_parameterised_type(dev):
    n = 9
    rng = W.SplitMix64(33)
    base = W.random_circuit(n, 80, 34, with_2x2=True)
    ops = base.copy()
    nparam = 0
    for i in range(len(ops)):
        if int(ops[i]["type"]) in (L.RX, L.RY, L.RZ, L.PHASE, L.CPHASE, L.MCPHASE):
            ops[i]["param"] = nparam % 7
            ops[i]["coeff"] = 0.5 + rng.uniform()
            nparam += 1
    params = np.array([rng.uniform() * 6.28 for _ in range(7)])
    obs_t = ([1 << q for q in range(n)] + [3, 0b101000], [1.0] * n + [0.25, -0.7], 0.3)
    v, g = _adjoint(dev, n, ops, params, obs_t)
    obs, keep = L.observable(*obs_t)
    vw, gw = O.adjoint(n, ops, params, obs)
    assert abs(v - vw) <= 1e-10
    assert np.max(np.abs(g - gw)) <= 1e-10


# ---------------------------------------------------------------- mid-circuit measurement
@pytest.mark.parametrize("n", [5, 12, 17])
def test_measure_and_reset_qubit_match_oracle(dev, n):
    rng = np.random.default_rng(n)
    for rep in range(4):
        ops = W.random_circuit(n, 20 * n, 6000 + 10 * n + rep)  # SWAPs relabel the qubit map
        want = O.run(n, ops)
        q = int(rng.integers(0, n))
        u = float(rng.random())
        for which in ("measure", "reset"):
            st = StateVector(n, dev)
            L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, None, None, 0, None))
            o = C.c_int32()
            p1 = C.c_double()
            fn = L.lib.qse_measure_qubit if which == "measure" else L.lib.qse_reset_qubit
            L.check(fn(st.handle, q, u, C.byref(o), C.byref(p1)))
            ref = want.copy()
            ro, rp1 = (O.measure_qubit if which == "measure" else O.reset_qubit)(ref, n, q, u)
            assert abs(p1.value - rp1) <= 1e-12
            if abs(u - rp1) > 1e-9:
                assert o.value == ro
                assert np.max(np.abs(st.download() - ref)) <= TOL


def test_execute_mid_circuit_measure_and_reset(dev):
    n = 11
    rng = np.random.default_rng(3)
    parts = [W.random_circuit(n, 60, 6100 + k) for k in range(4)]
    # MEASURE: target = qubit, control = result index (GateCommand::resultIdx)
    mid = [W.to_array([(L.MEASURE, 3, 1, -1, 0, 0.0, 1.0, (0.0,) * 8)]),
           W.to_array([(L.RESET_QUBIT, 7, 0, -1, 0, 0.0, 1.0, (0.0,) * 8)]),
           W.to_array([(L.MEASURE, 0, 0, -1, 0, 0.0, 1.0, (0.0,) * 8)])]
    ops = np.concatenate([parts[0], mid[0], parts[1], mid[1], parts[2], mid[2], parts[3]])
    u = rng.random(3)
    st = StateVector(n, dev)
    res = np.full(2, -1, dtype=np.int32)
    L.check(L.lib.qse_execute_mid(st.handle, L.dptr(ops), len(ops), None, 0, u.ctypes.data_as(L._pd), 3,
                                  res.ctypes.data_as(C.POINTER(C.c_int32)), 2))
    ref = O.run(n, parts[0])
    r1, _ = O.measure_qubit(ref, n, 3, u[0])
    ref = O.run_on(ref, n, parts[1])
    O.reset_qubit(ref, n, 7, u[1])
    ref = O.run_on(ref, n, parts[2])
    r0, _ = O.measure_qubit(ref, n, 0, u[2])
    ref = O.run_on(ref, n, parts[3])
    assert list(res) == [r0, r1]
    assert np.max(np.abs(st.download() - ref)) <= TOL
    # too few draws / a result index outside the array are rejected before anything runs
    with pytest.raises(L.QseError):
        L.check(L.lib.qse_execute_mid(st.handle, L.dptr(ops), len(ops), None, 0, u.ctypes.data_as(L._pd), 2,
                                      res.ctypes.data_as(C.POINTER(C.c_int32)), 2))
    with pytest.raises(L.QseError):
        L.check(L.lib.qse_execute_mid(st.handle, L.dptr(ops), len(ops), None, 0, u.ctypes.data_as(L._pd), 3,
                                      res.ctypes.data_as(C.POINTER(C.c_int32)), 1))


@pytest.mark.parametrize("n", [22, 24])
def test_streamed_passes_match_oracle(dev, n):
    """Pass-kernel mode 2: forward read+write passes over at least 2^10 tiles
    run as the persistent streamed kernel (bulk async copies into a three-slot
    shared-memory ring, two compute groups).  Random circuits over every gate
    and the H + RZ + QFT circuit against the oracle, and the same circuits
    through the one-CTA-per-tile kernels (which on these sizes take their group
    values from the precomputed table, so the phase products round in another
    order): equal within the amplitude tolerance."""
    L.check(L.lib.qse_ctx_set_jit(dev.handle, 2))
    try:
        for ops in (W.random_circuit(n, 12 * n, 7000 + n), W.hrz_qft(n, seed=2)):
            got, stats = run_gpu(dev, n, ops, fusion=True, k=12)
            assert np.max(np.abs(got - O.run(n, ops))) <= TOL
            L.check(L.lib.qse_ctx_set_jit(dev.handle, 1))
            classic, _ = run_gpu(dev, n, ops, fusion=True, k=12)
            L.check(L.lib.qse_ctx_set_jit(dev.handle, 2))
            assert np.max(np.abs(got - classic)) <= TOL
            # the state is the input of the next pass: an execute on top of it
            st = StateVector(n, dev)
            L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, None, None, 0, None))
            L.check(L.lib.qse_execute(st.handle, L.dptr(ops), len(ops), None, 0, None, None, 0, None))
            assert np.max(np.abs(st.download() - O.run(n, np.concatenate([ops, ops])))) <= TOL
    finally:
        L.check(L.lib.qse_ctx_set_jit(dev.handle, 1))
