"""Test-side access to the oracle (oracle/libqse_oracle.so) and, when it was
built in this checkout, to the reference sources compiled into oracle/_ref."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from quantumsimevo_b200.abi import OP_DTYPE, QseNoiseConfig, QseObservable

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_PATH = os.path.join(ROOT, "oracle", "libqse_oracle.so")
REF_CPU_PATH = os.path.join(ROOT, "oracle", "_ref", "libqse_ref_cpu.so")
REF_GPU_PATH = os.path.join(ROOT, "oracle", "_ref", "libqse_ref_gpu.so")
REF_PATCHED_PATH = os.path.join(ROOT, "oracle", "_ref", "libqse_ref_patched.so")

_vp, _u32, _u64, _sz, _d = C.c_void_p, C.c_uint32, C.c_uint64, C.c_size_t, C.c_double
_pd, _pu64 = C.POINTER(C.c_double), C.POINTER(C.c_uint64)


class OrcNoise(C.Structure):
    _fields_ = [("n", C.c_uint), ("bit", C.c_int32 * 64), ("phase", C.c_int32 * 64), ("rates", C.c_double * 16),
                ("mult", C.c_double), ("mode", C.c_int), ("mt_state", C.c_uint32 * 624), ("mt_idx", C.c_int),
                ("seed", C.c_uint64), ("draws", C.c_uint64)]


def _load_oracle():
    lib = C.CDLL(ORACLE_PATH)
    sigs = {
        "orc_init": ([_vp, C.c_uint], None),
        "orc_run": ([_vp, C.c_uint, _vp, _sz, _pd], C.c_int),
        "orc_cdf": ([_vp, C.c_uint, _pd], None),
        "orc_sample": ([_vp, C.c_uint, _pd, _sz, _pu64], None),
        "orc_sample_margin": ([_vp, C.c_uint, _pd, _sz, _pu64, _d], _sz),
        "orc_measure": ([_vp, C.c_uint, _d], _u64),
        "orc_mt_seed": ([_vp, _u32], None),
        "orc_mt_next": ([_vp], _u32),
        "orc_mt_canonical": ([_vp], _d),
        "orc_philox4x32_10": ([C.POINTER(_u32), C.POINTER(_u32), C.POINTER(_u32)], None),
        "orc_philox_uniform_pair": ([_u64, _u64, _pd, _pd], None),
        "orc_noise_init": ([C.POINTER(OrcNoise), C.c_uint, C.POINTER(QseNoiseConfig)], None),
        "orc_noise_accumulate": ([C.POINTER(OrcNoise), C.c_int, C.c_uint, _pd], C.c_int),
        "orc_measure_qubit": ([_vp, C.c_uint, C.c_uint, C.c_double, _pd], C.c_int),
        "orc_reset_qubit": ([_vp, C.c_uint, C.c_uint, C.c_double, _pd], C.c_int),
        "orc_execute": ([_vp, C.c_uint, _vp, _sz, _pd, C.POINTER(OrcNoise), _pd, _sz], C.c_int),
        "orc_expectation": ([_vp, C.c_uint, C.POINTER(QseObservable)], _d),
        "orc_adjoint": ([C.c_uint, _vp, _sz, _pd, _sz, C.POINTER(QseObservable), _pd], _d),
        "orc_param_shift": ([C.c_uint, _vp, _sz, _pd, _sz, C.POINTER(QseObservable), _pd], _d),
    }
    for name, (a, r) in sigs.items():
        f = getattr(lib, name)
        f.argtypes = a
        f.restype = r
    return lib


oracle = _load_oracle()


def ops_arr(ops):
    a = np.ascontiguousarray(ops)
    assert a.dtype == OP_DTYPE
    return a


def run(n, ops, params=None):
    """|0..0> then the ops; returns complex128 state."""
    st = np.zeros(1 << n, dtype=np.complex128)
    oracle.orc_init(st.ctypes.data_as(_vp), n)
    a = ops_arr(ops)
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
    rc = oracle.orc_run(st.ctypes.data_as(_vp), n, a.ctypes.data_as(_vp), len(a),
                        p.ctypes.data_as(_pd) if p is not None else None)
    assert rc == 0
    return st


def run_on(st, n, ops, params=None):
    st = np.ascontiguousarray(st, dtype=np.complex128).copy()
    a = ops_arr(ops)
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
    rc = oracle.orc_run(st.ctypes.data_as(_vp), n, a.ctypes.data_as(_vp), len(a),
                        p.ctypes.data_as(_pd) if p is not None else None)
    assert rc == 0
    return st


def execute_noisy(n, ops, cfg, uniforms=None, params=None, nz=None, st=None):
    if st is None:
        st = np.zeros(1 << n, dtype=np.complex128)
        oracle.orc_init(st.ctypes.data_as(_vp), n)
    if nz is None:
        nz = OrcNoise()
        oracle.orc_noise_init(C.byref(nz), n, C.byref(cfg))
    a = ops_arr(ops)
    u = None if uniforms is None else np.ascontiguousarray(uniforms, dtype=np.float64)
    p = None if params is None else np.ascontiguousarray(params, dtype=np.float64)
    rc = oracle.orc_execute(st.ctypes.data_as(_vp), n, a.ctypes.data_as(_vp), len(a),
                            p.ctypes.data_as(_pd) if p is not None else None, C.byref(nz),
                            u.ctypes.data_as(_pd) if u is not None else None, 0 if u is None else u.size)
    assert rc == 0, rc
    return st, nz


def sample(st, n, u):
    st = np.ascontiguousarray(st, dtype=np.complex128)
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.empty(u.size, dtype=np.uint64)
    oracle.orc_sample(st.ctypes.data_as(_vp), n, u.ctypes.data_as(_pd), u.size, out.ctypes.data_as(_pu64))
    return out


def sample_margin(st, n, u, ulps=4.0):
    """(outcomes, number of draws within `ulps` ulps of a cumulative boundary),
    one cumulative array (no copy of the state)."""
    st = np.ascontiguousarray(st, dtype=np.complex128)
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = np.empty(u.size, dtype=np.uint64)
    near = oracle.orc_sample_margin(st.ctypes.data_as(_vp), n, u.ctypes.data_as(_pd), u.size,
                                    out.ctypes.data_as(_pu64), float(ulps))
    assert near != C.c_size_t(-1).value, "oracle could not allocate the cumulative array"
    return out, int(near)


def measure_in_place(st, n, u):
    """orc_measure on st itself (collapsed in place; no copy of a large state)."""
    assert st.flags["C_CONTIGUOUS"] and st.dtype == np.complex128
    return int(oracle.orc_measure(st.ctypes.data_as(_vp), n, float(u)))


def cdf(st, n):
    st = np.ascontiguousarray(st, dtype=np.complex128)
    out = np.empty(1 << n, dtype=np.float64)
    oracle.orc_cdf(st.ctypes.data_as(_vp), n, out.ctypes.data_as(_pd))
    return out


def measure(st, n, u):
    st = np.ascontiguousarray(st, dtype=np.complex128).copy()
    idx = oracle.orc_measure(st.ctypes.data_as(_vp), n, float(u))
    return int(idx), st


def expectation(st, n, obs):
    st = np.ascontiguousarray(st, dtype=np.complex128)
    return oracle.orc_expectation(st.ctypes.data_as(_vp), n, C.byref(obs))


def adjoint(n, ops, params, obs):
    a = ops_arr(ops)
    p = np.ascontiguousarray(params, dtype=np.float64)
    g = np.zeros(p.size, dtype=np.float64)
    v = oracle.orc_adjoint(n, a.ctypes.data_as(_vp), len(a), p.ctypes.data_as(_pd), p.size, C.byref(obs),
                           g.ctypes.data_as(_pd))
    return v, g


def adjoint_job(args):
    """adjoint() on (n, ops, params, (zmasks, weights, constant)): picklable, for worker processes."""
    n, ops, params, (zm, w, c) = args
    z = np.ascontiguousarray(np.asarray(zm, dtype=np.uint64))
    wt = np.ascontiguousarray(np.asarray(w, dtype=np.float64))
    obs = QseObservable(len(z), z.ctypes.data_as(_pu64), wt.ctypes.data_as(_pd), float(c))
    return adjoint(n, ops, params, obs)


def param_shift(n, ops, params, obs):
    a = ops_arr(ops)
    p = np.ascontiguousarray(params, dtype=np.float64)
    g = np.zeros(p.size, dtype=np.float64)
    v = oracle.orc_param_shift(n, a.ctypes.data_as(_vp), len(a), p.ctypes.data_as(_pd), p.size, C.byref(obs),
                               g.ctypes.data_as(_pd))
    return v, g


def noise_decisions(n, ops, cfg):
    """Noise.cpp's per-gate draws and flip counts for a gate list, without a
    state (the decisions depend only on the gates and the draws)."""
    nz = OrcNoise()
    oracle.orc_noise_init(C.byref(nz), n, C.byref(cfg))
    for op in ops_arr(ops):
        oracle.orc_noise_accumulate(C.byref(nz), int(op["type"]), int(op["target"]), None)
    return list(nz.bit[:n]), list(nz.phase[:n])


def measure_qubit(st, n, q, u):
    """StateVector::measureQubit with the draw u; returns (outcome, prob1), st collapsed in place."""
    p = C.c_double()
    o = oracle.orc_measure_qubit(st.ctypes.data_as(_vp), n, q, u, C.byref(p))
    return o, p.value


def reset_qubit(st, n, q, u):
    p = C.c_double()
    o = oracle.orc_reset_qubit(st.ctypes.data_as(_vp), n, q, u, C.byref(p))
    return o, p.value


def philox_pair(seed, counter):
    a, b = C.c_double(), C.c_double()
    oracle.orc_philox_uniform_pair(seed, counter, C.byref(a), C.byref(b))
    return a.value, b.value


# ---------------- compiled reference (oracle/_ref) ----------------
def load_reference(gpu=False, patched=False):
    """The reference compiled into oracle/_ref: CPU backends, or (gpu) also its
    CUDA backend and this project's adapter, or (patched) the GPU build over a
    copy of the reference tree with the optional Circuit -> backend hooks."""
    path = REF_PATCHED_PATH if patched else REF_GPU_PATH if gpu else REF_CPU_PATH
    if not os.path.exists(path):
        return None
    lib = C.CDLL(path)
    sigs = {
        "ref_has_gpu": ([], C.c_int),
        "ref_set_quiet": ([C.c_int], None),
        "ref_set_backend": ([C.c_int], C.c_int),
        "ref_circuit_new": ([C.c_uint, C.c_int], _vp),
        "ref_circuit_free": ([_vp], None),
        "ref_circuit_add": ([_vp, _vp], C.c_int),
        "ref_circuit_add_many": ([_vp, _vp, _sz], C.c_int),
        "ref_circuit_execute": ([_vp, C.c_int], None),
        "ref_circuit_reset": ([_vp], None),
        "ref_circuit_state": ([_vp, _vp], None),
        "ref_circuit_measure": ([_vp], _u64),
        "ref_circuit_sample": ([_vp, C.c_int, _pu64], None),
        "ref_noise_run": ([C.c_uint, C.c_uint, _d, C.POINTER(C.c_int), C.POINTER(C.c_uint), _sz, _vp, _pu64, _pu64],
                          None),
        "ref_std_uniforms": ([C.c_uint, _sz, _pd], None),
        "ref_backend_new": ([C.c_int], _vp),
        "ref_backend_free": ([_vp], None),
        "ref_statevector_new": ([C.c_uint], _vp),
        "ref_statevector_free": ([_vp], None),
        "ref_backend_apply": ([_vp, _vp, _vp, _sz], C.c_int),
        "ref_backend_flush": ([_vp], None),
        "ref_backend_mark_host_dirty": ([_vp], None),
        "ref_statevector_get": ([_vp, _vp], None),
        "ref_statevector_set": ([_vp, _vp], None),
        "ref_statevector_measure_qubit": ([_vp, C.c_uint], C.c_int),
        "ref_statevector_measure": ([_vp], _u64),
        "ref_statevector_sample": ([_vp, C.c_int, _pu64], None),
        "ref_statevector_reset": ([_vp], None),
        "ref_device_synchronize": ([], C.c_int),
        "ref_statevector_reset_qubit": ([_vp, C.c_uint], None),
        "ref_playground_build": ([_vp, C.c_int, C.c_int, C.c_int], C.c_int),
        "ref_tsp_ising": ([_pd, C.c_uint, _d, _d, C.c_int, C.c_int, _pd, C.POINTER(C.c_uint), _pd, C.c_uint,
                           C.POINTER(C.c_uint)], C.c_int),
    }
    if gpu or patched:
        sigs["ref_b200_sample"] = ([_vp, _vp, _pd, _sz, _pu64], C.c_int)
        sigs["ref_b200_measure"] = ([_vp, _vp, _d, _pu64], C.c_int)
        sigs["ref_b200_kernel_launches"] = ([], _u64)
    if patched:
        sigs["ref_inject_uniforms"] = ([_pd, _sz], None)
    for name, (a, r) in sigs.items():
        f = getattr(lib, name)
        f.argtypes = a
        f.restype = r
    return lib


def ref_playground(ref, which, n, target=0, iterations=0):
    """State from the reference playground's own builder (0 = runQFT's circuit, 1 = runIQFT's,
    2 = Grover::createGroverCircuit) on the reference Circuit with the scalar backend."""
    assert ref.ref_set_backend(0) == 0
    h = ref.ref_circuit_new(n, 0)
    assert ref.ref_playground_build(h, which, target, iterations) == 0
    ref.ref_circuit_execute(h, 0)
    out = np.empty(1 << n, dtype=np.complex128)
    ref.ref_circuit_state(h, out.ctypes.data_as(_vp))
    ref.ref_circuit_free(h)
    return out


def ref_run(ref, n, ops, backend=0):
    """Reference Circuit (scalar by default): queue ops, execute, return the state."""
    assert ref.ref_set_backend(backend) == 0
    h = ref.ref_circuit_new(n, 0)
    a = ops_arr(ops)
    assert ref.ref_circuit_add_many(h, a.ctypes.data_as(_vp), len(a)) == 0
    ref.ref_circuit_execute(h, 0)
    out = np.empty(1 << n, dtype=np.complex128)
    ref.ref_circuit_state(h, out.ctypes.data_as(_vp))
    ref.ref_circuit_free(h)
    ref.ref_set_backend(0)
    return out
