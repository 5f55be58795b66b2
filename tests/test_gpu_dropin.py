"""The reference's own Circuit / StateVector / Noise (compiled from its sources
into oracle/_ref) running on this project's drop-in backend
CircuitUnitaryOperationB200, against the same reference code on its scalar
backend; plus the torch.autograd binding."""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle_ffi as O
from quantumsimevo_b200 import _lib as L
from quantumsimevo_b200 import workloads as W
from quantumsimevo_b200.autograd import ParametrizedCircuit, QuantumLayer

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    r = O.load_reference(gpu=True)
    if r is None:
        pytest.skip("oracle/_ref/libqse_ref_gpu.so not built")
    r.ref_set_quiet(1)
    return r


@pytest.mark.parametrize("n", [1, 3, 6, 10, 14])
def test_reference_circuit_on_b200_adapter(ref, n):
    for rep in range(2):
        ops = W.random_circuit(n, 30 * n + 10, 8000 + 11 * n + rep, with_2x2=False)
        want = O.ref_run(ref, n, ops, backend=0)     # reference Circuit, scalar backend
        got = O.ref_run(ref, n, ops, backend=3)      # reference Circuit, CircuitUnitaryOperationB200
        assert np.max(np.abs(got - want)) <= 1e-12


def test_reference_gpu_backend_rebuilt_for_sm100(ref):
    # the reference's own CUDA backend compiled for sm_100a (the plain-kernel baseline)
    n = 12
    ops = W.random_circuit(n, 300, 81, with_2x2=False)
    want = O.ref_run(ref, n, ops, backend=0)
    got = O.ref_run(ref, n, ops, backend=2)
    assert np.max(np.abs(got - want)) <= 1e-12


def test_reference_noise_through_adapter(ref):
    # Circuit(N, true): Noise(N, 42, 1) draws from mt19937 and applies X/Z through the backend
    n = 9
    ops = W.random_circuit(n, 400, 82, with_2x2=False)
    outs = []
    for backend in (0, 3):
        assert ref.ref_set_backend(backend) == 0
        h = ref.ref_circuit_new(n, 1)
        a = np.ascontiguousarray(ops)
        ref.ref_circuit_add_many(h, a.ctypes.data_as(C.c_void_p), len(a))
        ref.ref_circuit_execute(h, 0)
        ref.ref_circuit_execute(h, 0)   # the queue is replayed and the noise re-applied
        st = np.empty(1 << n, dtype=np.complex128)
        ref.ref_circuit_state(h, st.ctypes.data_as(C.c_void_p))
        ref.ref_circuit_free(h)
        outs.append(st)
    ref.ref_set_backend(0)
    assert np.max(np.abs(outs[0] - outs[1])) <= 1e-12


def test_adapter_flush_and_host_dirty(ref):
    # per-gate through the backend object: markHostDirty re-uploads host edits
    n = 8
    be = ref.ref_backend_new(3)
    sv = ref.ref_statevector_new(n)
    ops = W.random_circuit(n, 60, 83, with_2x2=True)
    a = np.ascontiguousarray(ops)
    assert ref.ref_backend_apply(be, sv, a.ctypes.data_as(C.c_void_p), len(a)) == 0
    ref.ref_backend_flush(be)
    st = np.empty(1 << n, dtype=np.complex128)
    ref.ref_statevector_get(sv, st.ctypes.data_as(C.c_void_p))
    assert np.max(np.abs(st - O.run(n, ops))) <= 1e-12
    # edit on the host, mark dirty, apply more gates
    edited = np.roll(st, 3)
    ref.ref_statevector_set(sv, edited.ctypes.data_as(C.c_void_p))
    ref.ref_backend_mark_host_dirty(be)
    more = np.ascontiguousarray(W.random_circuit(n, 20, 84, with_2x2=True))
    assert ref.ref_backend_apply(be, sv, more.ctypes.data_as(C.c_void_p), len(more)) == 0
    ref.ref_backend_flush(be)
    ref.ref_statevector_get(sv, st.ctypes.data_as(C.c_void_p))
    assert np.max(np.abs(st - O.run_on(edited, n, more))) <= 1e-12
    ref.ref_statevector_free(sv)
    ref.ref_backend_free(be)


def test_adapter_sample_and_measure_extensions(ref):
    # CircuitUnitaryOperationB200::sample / measure with injected uniforms: the
    # outcomes StateVector::sample / measure give for the same draws, and the
    # collapse lands on the host at the next flush
    n = 12
    be = ref.ref_backend_new(3)
    sv = ref.ref_statevector_new(n)
    ops = np.ascontiguousarray(W.random_circuit(n, 150, 85, with_2x2=True))
    assert ref.ref_backend_apply(be, sv, ops.ctypes.data_as(C.c_void_p), len(ops)) == 0
    ref.ref_backend_flush(be)
    st = np.empty(1 << n, dtype=np.complex128)
    ref.ref_statevector_get(sv, st.ctypes.data_as(C.c_void_p))
    u = np.random.default_rng(85).random(3000)
    out = np.empty(len(u), dtype=np.uint64)
    assert ref.ref_b200_sample(be, sv, u.ctypes.data_as(O._pd), len(u), out.ctypes.data_as(O._pu64)) == 0
    assert np.array_equal(out, O.sample(st, n, u))
    idx = np.zeros(1, dtype=np.uint64)
    assert ref.ref_b200_measure(be, sv, 0.437, idx.ctypes.data_as(O._pu64)) == 0
    want_idx, want_st = O.measure(st, n, 0.437)
    assert int(idx[0]) == want_idx
    ref.ref_backend_flush(be)
    ref.ref_statevector_get(sv, st.ctypes.data_as(C.c_void_p))
    assert np.array_equal(st, want_st)
    ref.ref_statevector_free(sv)
    ref.ref_backend_free(be)


def test_torch_autograd_matches_oracle_and_fd():
    n = 10
    ops, params, edges, obs_t = W.qaoa_maxcut(n, 2, seed=90)
    pc = ParametrizedCircuit(n, ops, *obs_t)
    layer = QuantumLayer(pc, params)
    val = layer()
    val.backward()
    obs, keep = L.observable(*obs_t)
    vw, gw = O.adjoint(n, ops, params, obs)
    assert abs(val.item() - vw) <= 1e-10
    assert np.max(np.abs(layer.params.grad.numpy() - gw)) <= 1e-10
    # central finite differences, h = 1e-6: round-off limits agreement to ~1e-7
    h = 1e-6
    for k in range(len(params)):
        pp, pm = params.copy(), params.copy()
        pp[k] += h
        pm[k] -= h
        fd = (pc.value(pp) - pc.value(pm)) / (2 * h)
        assert abs(fd - gw[k]) <= 1e-7 * max(1.0, abs(gw[k]))
    # no-grad forward
    with torch.no_grad():
        v2 = pc.expectation(torch.tensor(params))
    assert abs(v2.item() - vw) <= 1e-10


def test_python_circuit_parameters_expectation_gradient_measure_qubit():
    """The Python surface beyond the reference's pybind module: parameterised
    gates, execute(params), expectation, gradient (adjoint) and measure_qubit,
    each against the oracle."""
    import numpy as np

    import oracle_ffi as O
    from quantumsimevo_b200 import _lib as L
    from quantumsimevo_b200.circuit import Circuit
    n = 9
    c = Circuit(n, seed=1)
    for q in range(n):
        c.hadamard(q)
    for layer in range(2):
        for q in range(n - 1):
            c.cphase(0.0, q, q + 1, param=layer, coeff=-2.0)
        for q in range(n):
            c.rotate_x(0.1, q, param=2 + layer, coeff=2.0)
        c.rotate_z(0.3, layer, param=4)
        c.mcphase(0.2, [0, 1], 5, param=4, coeff=0.5)
    params = np.array([0.3, 1.1, 0.7, 0.2, 0.9])
    zm, wt, const = [1 << q for q in range(n)] + [0b11], [0.5] * n + [-1.0], 0.25
    c.execute(params=params)
    want = O.run(n, c.ops, params)
    assert np.max(np.abs(c.get_state_vector() - want)) <= 1e-12
    obs, keep = L.observable(zm, wt, const)
    assert abs(c.expectation(zm, wt, const) - O.expectation(want, n, obs)) <= 1e-12
    v, g = c.gradient(params, zm, wt, const)
    vw, gw = O.adjoint(n, c.ops, params, obs)
    assert abs(v - vw) <= 1e-10 and np.max(np.abs(g - gw)) <= 1e-10
    c.reset()
    c.hadamard(2)
    c.cnot(2, 6)
    c.execute()
    o = c.measure_qubit(6, uniform=0.25)
    st = c.get_state_vector()
    assert o in (0, 1)
    idx = 1 << 2 | 1 << 6 if o else 0
    assert abs(abs(st[idx]) - 1.0) <= 1e-12


@pytest.fixture(scope="module")
def ref_patched():
    r = O.load_reference(patched=True)
    if r is None:
        pytest.skip("oracle/_ref/libqse_ref_patched.so not built")
    r.ref_set_quiet(1)
    return r


@pytest.mark.parametrize("n", [5, 12, 16])
def test_patched_reference_circuit_takes_the_fused_path(ref_patched, n):
    """The reference's own Circuit compiled over a copy of its tree whose
    interface declares the optional hooks (oracle/patch_reference.py):
    Circuit::execute hands the whole queue to CircuitUnitaryOperationB200::
    executeProgram -> qse_execute (fused passes), and Circuit::sample /
    Circuit::measure hand their draws to the device sampler.  Against the same
    Circuit on the scalar backend, whose hooks decline: amplitudes <= 1e-12
    (SWAP and MCPHASE included); the execute launches a few passes, not one
    kernel per gate; sample / measure give the oracle's outcomes for the
    injected draws on the device state."""
    r = ref_patched
    ops = W.random_circuit(n, 40 * n, 9100 + n, with_2x2=False)
    assert np.any(ops["type"] == L.SWAP) and np.any(ops["type"] == L.MCPHASE)
    want = O.ref_run(r, n, ops, backend=0)
    assert r.ref_set_backend(3) == 0
    h = r.ref_circuit_new(n, 0)
    a = np.ascontiguousarray(ops)
    assert r.ref_circuit_add_many(h, a.ctypes.data_as(C.c_void_p), len(a)) == 0
    k0 = r.ref_b200_kernel_launches()
    r.ref_circuit_execute(h, 0)
    launches = r.ref_b200_kernel_launches() - k0
    got = np.empty(1 << n, dtype=np.complex128)
    r.ref_circuit_state(h, got.ctypes.data_as(C.c_void_p))
    assert np.max(np.abs(got - want)) <= 1e-12
    assert launches < len(ops) / 4, (launches, len(ops))
    u = np.random.default_rng(n).random(2000)
    r.ref_inject_uniforms(u.ctypes.data_as(O._pd), u.size)
    out = np.empty(u.size, dtype=np.uint64)
    r.ref_circuit_sample(h, u.size, out.ctypes.data_as(O._pu64))
    assert np.array_equal(out, O.sample(got, n, u))
    um = np.array([0.41421356])
    r.ref_inject_uniforms(um.ctypes.data_as(O._pd), 1)
    idx = r.ref_circuit_measure(h)
    want_idx, collapsed = O.measure(got, n, um[0])
    assert idx == want_idx
    after = np.empty(1 << n, dtype=np.complex128)
    r.ref_circuit_state(h, after.ctypes.data_as(C.c_void_p))
    assert np.array_equal(after, collapsed)
    r.ref_circuit_free(h)
    r.ref_set_backend(0)
