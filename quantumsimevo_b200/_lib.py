"""ctypes binding of libqse_b200.so (the C ABI declared in include/qse_b200.h).

The shared library is built in-tree (``quantumsimevo_b200/libqse_b200.so``).
There is no fallback: if the library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libqse_b200.so")

# gate types: GateType numbering (QuantumSimEvo/Structurs.h:10) + GATE2X2
IDENTITY, X, Y, Z, H, PHASE, RX, RY, RZ, CNOT, CPHASE, MCPHASE, SWAP, MEASURE, RESET_QUBIT, GATE2X2 = range(16)
GATE_NAMES = {IDENTITY: "I", X: "X", Y: "Y", Z: "Z", H: "H", PHASE: "PHASE", RX: "RX", RY: "RY", RZ: "RZ",
              CNOT: "CNOT", CPHASE: "CPHASE", MCPHASE: "MCPHASE", SWAP: "SWAP", GATE2X2: "U"}

RNG_PHILOX, RNG_MT19937, RNG_INJECTED = 0, 1, 2

OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "QUBIT", 3: "OOM", 4: "CUDA", 5: "SIZE", 6: "UNSUPPORTED",
                7: "TIMEOUT", 8: "STATE"}

# numpy mirror of struct qse_op (104 bytes)
OP_DTYPE = np.dtype([("type", "<i4"), ("target", "<u4"), ("control", "<u4"), ("param", "<i4"),
                     ("controls", "<u8"), ("theta", "<f8"), ("coeff", "<f8"), ("m", "<f8", (8,))])
assert OP_DTYPE.itemsize == 104


class QseOp(C.Structure):
    _fields_ = [("type", C.c_int32), ("target", C.c_uint32), ("control", C.c_uint32), ("param", C.c_int32),
                ("controls", C.c_uint64), ("theta", C.c_double), ("coeff", C.c_double), ("m", C.c_double * 8)]


class QseObservable(C.Structure):
    _fields_ = [("nterms", C.c_size_t), ("zmask", C.POINTER(C.c_uint64)), ("weight", C.POINTER(C.c_double)),
                ("constant", C.c_double)]


class QseNoiseConfig(C.Structure):
    _fields_ = [("enabled", C.c_int32), ("rng_mode", C.c_int32), ("seed", C.c_uint64), ("multiplier", C.c_double),
                ("rates", C.c_double * 16)]


class QseExecStats(C.Structure):
    _fields_ = [("gates", C.c_uint64), ("passes", C.c_uint64), ("kernels", C.c_uint64), ("noisy_gates", C.c_uint64)]


class QseBatchCircuit(C.Structure):
    _fields_ = [("nqubits", C.c_uint32), ("nops", C.c_size_t), ("ops", C.c_void_p), ("nparams", C.c_size_t),
                ("obs", QseObservable)]


class QseBatchConfig(C.Structure):
    _fields_ = [("threads", C.c_uint32), ("reg_bits", C.c_uint32), ("max_gates", C.c_uint32),
                ("chain_tiles", C.c_uint32), ("ctas_per_sm", C.c_uint32), ("grad_slots", C.c_uint32),
                ("wide_regs", C.c_uint32)]


class QseBatchStats(C.Structure):
    _fields_ = [("passes", C.c_uint64), ("items", C.c_uint64), ("tile_visits", C.c_uint64),
                ("hbm_bytes", C.c_uint64), ("occurrences", C.c_uint64), ("grid", C.c_uint32),
                ("smem_bytes", C.c_uint32), ("last_ms", C.c_double), ("plan_ms", C.c_double)]


assert C.sizeof(QseOp) == 104


class QseError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"qse error {STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`"
                          " (or `make -C quantumsimevo_b200/csrc`)")
    return C.CDLL(LIB_PATH)


lib = _load()

_vp, _u32, _u64, _i32, _sz, _d = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32, C.c_size_t, C.c_double
_pd, _pu64 = C.POINTER(C.c_double), C.POINTER(C.c_uint64)

_SIGS = {
    "qse_last_error": ([], C.c_char_p),
    "qse_version": ([], C.c_char_p),
    "qse_ctx_create": ([C.c_int, C.POINTER(_vp)], C.c_int),
    "qse_ctx_destroy": ([_vp], C.c_int),
    "qse_ctx_synchronize": ([_vp], C.c_int),
    "qse_ctx_set_fusion": ([_vp, C.c_int, C.c_int, C.c_int], C.c_int),
    "qse_ctx_set_sample_mode": ([_vp, C.c_int], C.c_int),
    "qse_ctx_kernel_launches": ([_vp], _u64),
    "qse_ctx_record": ([_vp, C.c_int], C.c_int),
    "qse_ctx_elapsed": ([_vp, C.c_int, C.c_int, C.POINTER(C.c_float)], C.c_int),
    "qse_ctx_time_passes": ([_vp, C.c_int], C.c_int),
    "qse_ctx_pass_times": ([_vp, _pu64, _pd], C.c_int),
    "qse_ctx_pass_time_list": ([_vp, _pd, _sz, C.POINTER(_sz)], C.c_int),
    "qse_sample_device": ([_vp, _vp, _sz, _u64, _vp], C.c_int),
    "qse_state_create": ([_vp, _u32, C.POINTER(_vp)], C.c_int),
    "qse_state_destroy": ([_vp], C.c_int),
    "qse_state_qubits": ([_vp], _u32),
    "qse_state_reset": ([_vp], C.c_int),
    "qse_state_upload": ([_vp, _vp], C.c_int),
    "qse_state_download": ([_vp, _vp], C.c_int),
    "qse_state_download_range": ([_vp, _u64, _u64, _vp], C.c_int),
    "qse_state_device_ptr": ([_vp, C.POINTER(_vp)], C.c_int),
    "qse_state_qubit_map": ([_vp, C.POINTER(_u32)], C.c_int),
    "qse_state_canonicalize": ([_vp], C.c_int),
    "qse_apply_gate2x2": ([_vp, _pd, _u32], C.c_int),
    "qse_apply_cnot": ([_vp, _u32, _u32], C.c_int),
    "qse_apply_x": ([_vp, _u32], C.c_int),
    "qse_apply_y": ([_vp, _u32], C.c_int),
    "qse_apply_z": ([_vp, _u32], C.c_int),
    "qse_apply_phase": ([_vp, _u32, _d], C.c_int),
    "qse_apply_rx": ([_vp, _u32, _d], C.c_int),
    "qse_apply_ry": ([_vp, _u32, _d], C.c_int),
    "qse_apply_rz": ([_vp, _u32, _d], C.c_int),
    "qse_apply_h": ([_vp, _u32], C.c_int),
    "qse_apply_cphase": ([_vp, _u32, _u32, _d], C.c_int),
    "qse_apply_mcphase": ([_vp, C.POINTER(_u32), _sz, _u32, _d], C.c_int),
    "qse_apply_swap": ([_vp, _u32, _u32], C.c_int),
    "qse_noise_create": ([_vp, _u32, C.POINTER(QseNoiseConfig), C.POINTER(_vp)], C.c_int),
    "qse_noise_destroy": ([_vp], C.c_int),
    "qse_noise_reset_stats": ([_vp], C.c_int),
    "qse_noise_counts": ([_vp, C.POINTER(_i32), C.POINTER(_i32)], C.c_int),
    "qse_execute": ([_vp, _vp, _sz, _pd, _sz, _vp, _pd, _sz, C.POINTER(QseExecStats)], C.c_int),
    "qse_plan_describe": ([_u32, _vp, _sz, _pd, _sz, _u32, _u32, C.c_char_p, _sz, C.POINTER(_sz)], C.c_int),
    "qse_sample": ([_vp, _pd, _sz, _u64, _pu64], C.c_int),
    "qse_measure": ([_vp, _d, _pu64], C.c_int),
    "qse_measure_qubit": ([_vp, _u32, _d, C.POINTER(_i32), _pd], C.c_int),
    "qse_reset_qubit": ([_vp, _u32, _d, C.POINTER(_i32), _pd], C.c_int),
    "qse_execute_mid": ([_vp, _vp, _sz, _pd, _sz, _pd, _sz, C.POINTER(_i32), _sz], C.c_int),
    "qse_total_probability": ([_vp, _pd], C.c_int),
    "qse_expectation": ([_vp, C.POINTER(QseObservable), _pd], C.c_int),
    "qse_adjoint": ([_vp, _vp, _sz, _pd, _sz, C.POINTER(QseObservable), _pd, _pd], C.c_int),
    "qse_batch_create": ([_vp, C.POINTER(QseBatchCircuit), _sz, C.POINTER(_vp)], C.c_int),
    "qse_batch_destroy": ([_vp], C.c_int),
    "qse_batch_run": ([_vp, _pd, _pd, _pd], C.c_int),
    "qse_batch_run_device": ([_vp, _vp, _vp, _vp], C.c_int),
    "qse_batch_total_params": ([_vp, C.POINTER(_sz)], C.c_int),
    "qse_batch_autotune": ([_vp, C.c_char_p], C.c_int),
    "qse_batch_use_graph": ([_vp, C.c_int], C.c_int),
    "qse_batch_set_config": ([_vp, C.POINTER(QseBatchConfig)], C.c_int),
    "qse_batch_get_config": ([_vp, C.POINTER(QseBatchConfig)], C.c_int),
    "qse_batch_get_stats": ([_vp, C.POINTER(QseBatchStats)], C.c_int),
}

for _name, (_args, _res) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = _res


def check(status: int) -> None:
    if status != OK:
        msg = lib.qse_last_error()
        raise QseError(status, msg.decode() if msg else "")


def dptr(a: np.ndarray):
    """ctypes pointer to a numpy array's data (array must stay alive)."""
    return a.ctypes.data_as(C.c_void_p)


def as_ops(ops) -> np.ndarray:
    """Coerce a sequence of QseOp / tuples / an OP_DTYPE array to a contiguous OP_DTYPE array."""
    if isinstance(ops, np.ndarray) and ops.dtype == OP_DTYPE:
        return np.ascontiguousarray(ops)
    arr = np.zeros(len(ops), dtype=OP_DTYPE)
    for i, o in enumerate(ops):
        arr[i] = o
    return arr


def make_op(type_: int, target: int = 0, control: int = 0, theta: float = 0.0, controls=(), param: int = -1,
            coeff: float = 1.0, m=None):
    mask = 0
    for c in controls:
        mask |= 1 << int(c)
    mm = tuple(m) if m is not None else (0.0,) * 8
    return (type_, target, control, param, mask, theta, coeff, mm)


def observable(zmasks, weights, constant=0.0):
    """Returns (QseObservable, keepalive) for Z-string terms."""
    z = np.ascontiguousarray(np.asarray(zmasks, dtype=np.uint64))
    w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64))
    obs = QseObservable(len(z), z.ctypes.data_as(_pu64), w.ctypes.data_as(_pd), float(constant))
    return obs, (z, w)


def default_noise_config(enabled=True, rng_mode=RNG_PHILOX, seed=42, multiplier=1.0, rates=None) -> QseNoiseConfig:
    """Noise(N, 42, 1) defaults (Noise.cpp:10-18); -1 = type not in the error-rate map."""
    r = [-1.0] * 16
    if rates is None:
        for t, p in ((X, 1e-3), (Y, 1e-3), (Z, 1e-3), (H, 2e-3), (CNOT, 5e-3), (PHASE, 1e-3), (RX, 1e-3),
                     (RY, 1e-3), (RZ, 1e-3)):
            r[t] = p
    else:
        for t, p in rates.items():
            r[t] = p
    cfg = QseNoiseConfig()
    cfg.enabled = 1 if enabled else 0
    cfg.rng_mode = rng_mode
    cfg.seed = seed
    cfg.multiplier = multiplier
    for i in range(16):
        cfg.rates[i] = r[i]
    return cfg

for _name, (_args, _res) in {
    "qse_ctx_set_jit": ([_vp, C.c_int], C.c_int),
    "qse_sampler_stats": ([_vp, C.POINTER(_u32)], C.c_int),
    "qse_expectation_noalloc": ([_vp, C.POINTER(QseObservable), _pd], C.c_int),
    "qse_plan_compile": ([_u32, _vp, _sz, _pd, _sz, _u32, C.c_int, C.POINTER(_sz)], C.c_int),
}.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = _res
