"""ctypes binding of libqse_b200.so (the C ABI declared in include/qse_b200.h).

The shared library is built in-tree (``quantumsimevo_b200/libqse_b200.so``).
There is no fallback: if the library is missing, importing this module raises.
The plain-data side of the ABI (gate numbers, structures, op arrays) lives in
``abi`` and is re-exported here.
"""
from __future__ import annotations

import ctypes as C
import os

from .abi import *  # noqa: F401,F403
from .abi import OK, QseBatchCircuit, QseBatchConfig, QseBatchStats, QseError, QseExecStats, QseNoiseConfig, QseObservable

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libqse_b200.so")


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
    "qse_batch_set_wait_limit": ([_vp, _u32], C.c_int),
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


for _name, (_args, _res) in {
    "qse_ctx_set_jit": ([_vp, C.c_int], C.c_int),
    "qse_sampler_stats": ([_vp, C.POINTER(_u32)], C.c_int),
    "qse_expectation_noalloc": ([_vp, C.POINTER(QseObservable), _pd], C.c_int),
    "qse_plan_compile": ([_u32, _vp, _sz, _pd, _sz, _u32, C.c_int, C.POINTER(_sz)], C.c_int),
}.items():
    _f = getattr(lib, _name)
    _f.argtypes = _args
    _f.restype = _res
