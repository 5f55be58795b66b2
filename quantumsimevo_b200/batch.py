"""Batched forward expectation + adjoint gradient of many parameterised circuits
(qse_batch_* in include/qse_b200.h): one persistent kernel per run, replayed as
a CUDA graph.

No reference counterpart: QuantumSimEvo evaluates one Circuit at a time
(QuantumSimEvo/Circuit.cpp:64-120).  Gate semantics are the reference's
(QuantumSimEvo/CircuitUnitaryOperation.cpp); the gradient of a parameterised
gate occurrence is d<O>/d(angle) times the op's coefficient, summed per
parameter.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from ._lib import check, lib
from .circuit import Device


@dataclass
class BatchConfig:
    threads: int = 256      # CTA size (power of two, 32..512)
    reg_bits: int = 3       # 2^reg_bits amplitudes per thread; tile qubits = log2(threads) + reg_bits
    max_gates: int = 0      # non-diagonal gates per pass, 0 = no cap
    chain_tiles: int = 1    # circuits with <= this many tiles run start to end in one CTA
    ctas_per_sm: int = 0    # 0 = as many as fit
    grad_slots: int = 0     # gradient slots per pass, 0 = no cap
    wide_regs: int = 0      # 1: up to 255 registers per thread (threads <= 256); 0: 128


class Batch:
    """circuits: iterable of (nqubits, ops, nparams, (zmasks, weights, constant)).

    ops is an OP_DTYPE array whose ``param`` fields index the circuit's own
    parameters; the observable is constant + sum_t weight[t] * Z-string(zmask[t]).
    """

    def __init__(self, circuits, device: Device | None = None):
        self.device = device or Device.default()
        self._keep = []
        circs = list(circuits)
        arr = (L.QseBatchCircuit * max(1, len(circs)))()
        self.nparams = []
        for i, (n, ops, npar, obs) in enumerate(circs):
            ops = L.as_ops(ops)
            z = np.ascontiguousarray(np.asarray(obs[0], dtype=np.uint64))
            w = np.ascontiguousarray(np.asarray(obs[1], dtype=np.float64))
            self._keep += [ops, z, w]
            arr[i].nqubits = int(n)
            arr[i].nops = len(ops)
            arr[i].ops = ops.ctypes.data_as(C.c_void_p)
            arr[i].nparams = int(npar)
            arr[i].obs.nterms = len(z)
            arr[i].obs.zmask = z.ctypes.data_as(C.POINTER(C.c_uint64))
            arr[i].obs.weight = w.ctypes.data_as(C.POINTER(C.c_double))
            arr[i].obs.constant = float(obs[2])
            self.nparams.append(int(npar))
        h = C.c_void_p()
        check(lib.qse_batch_create(self.device.handle, arr, len(circs), C.byref(h)))
        self.handle = h
        self.ncircuits = len(circs)
        self.offsets = np.concatenate([[0], np.cumsum(self.nparams)]).astype(np.int64)
        total = C.c_size_t()
        check(lib.qse_batch_total_params(h, C.byref(total)))
        self.total_params = int(total.value)

    # configuration ---------------------------------------------------------
    @property
    def config(self) -> BatchConfig:
        c = L.QseBatchConfig()
        check(lib.qse_batch_get_config(self.handle, C.byref(c)))
        return BatchConfig(c.threads, c.reg_bits, c.max_gates, c.chain_tiles, c.ctas_per_sm, c.grad_slots,
                           c.wide_regs)

    @config.setter
    def config(self, cfg: BatchConfig) -> None:
        c = L.QseBatchConfig(cfg.threads, cfg.reg_bits, cfg.max_gates, cfg.chain_tiles, cfg.ctas_per_sm,
                             cfg.grad_slots, cfg.wide_regs)
        check(lib.qse_batch_set_config(self.handle, C.byref(c)))

    def autotune(self, cache_path: str | None = None) -> BatchConfig:
        check(lib.qse_batch_autotune(self.handle, cache_path.encode() if cache_path else None))
        return self.config

    def set_wait_limit(self, polls: int = 0) -> None:
        """Polls before a dependency wait of the persistent kernel gives up
        (the run then raises QseError with status TIMEOUT); 0 = the default."""
        check(lib.qse_batch_set_wait_limit(self.handle, int(polls)))

    def use_graph(self, enabled: bool = True) -> None:
        check(lib.qse_batch_use_graph(self.handle, 1 if enabled else 0))

    def stats(self) -> dict:
        s = L.QseBatchStats()
        check(lib.qse_batch_get_stats(self.handle, C.byref(s)))
        return {f: getattr(s, f) for f, _ in L.QseBatchStats._fields_}

    # runs --------------------------------------------------------------------
    def run(self, params):
        """params: concatenation of every circuit's parameters.  Returns
        (values[ncircuits], grads like params)."""
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
        if p.size != self.total_params:
            raise ValueError(f"expected {self.total_params} parameters, got {p.size}")
        values = np.zeros(self.ncircuits, dtype=np.float64)
        grads = np.zeros(max(1, self.total_params), dtype=np.float64)
        check(lib.qse_batch_run(self.handle, p.ctypes.data_as(L._pd), values.ctypes.data_as(L._pd),
                                grads.ctypes.data_as(L._pd)))
        return values, grads[: self.total_params]

    def run_device(self, d_params: int, d_values: int, d_grads: int) -> None:
        """Device pointers (e.g. torch tensor.data_ptr()); asynchronous on the device's stream."""
        check(lib.qse_batch_run_device(self.handle, C.c_void_p(d_params), C.c_void_p(d_values),
                                       C.c_void_p(d_grads)))

    def split(self, flat):
        """Per-circuit views of a flat parameter / gradient vector."""
        return [flat[self.offsets[i]:self.offsets[i + 1]] for i in range(self.ncircuits)]

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            lib.qse_batch_destroy(h)
            self.handle = None
