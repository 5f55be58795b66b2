"""Plain-data side of the C ABI (include/qse_b200.h): gate-type numbers,
the numpy mirror of struct qse_op, the ctypes structures and the small
helpers that build them.  Importing this module loads no native library, so
workload generators and test checkers can use it on machines (or in
processes) that must not map libqse_b200.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

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


_pd, _pu64 = C.POINTER(C.c_double), C.POINTER(C.c_uint64)


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
