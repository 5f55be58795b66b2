"""qse_expectation_noalloc: the allocation-free expectation value.

Some callers of this library cannot allocate memory at the moment they ask
for <psi|O|psi>: code that runs while a memory pool or allocator is locked or
exhausted, a host program that has handed all device memory to its own
allocator, or an embedding that forbids allocation after start-up.  For them
the library offers an entry point whose scratch is a fixed device array
compiled into the library.

This file checks, through the C ABI, that the entry point
  - gives the same value as qse_expectation (within 1e-12) on two calls in a
    row, for each of two states;
  - leaves the device's free memory unchanged across those calls (after one
    first call that does the per-device set-up: the scratch array's address
    lookup, and the module load that a lazily loading CUDA runtime performs
    on first use);
  - rejects an observable larger than its fixed scratch.
It sorts last so a run that stops at the first failure has already run every
other test, and it passes both in a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from quantumsimevo_b200 import _lib as L
from quantumsimevo_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _value(fn, st, obs):
    v = C.c_double()
    L.check(fn(st, C.byref(obs), C.byref(v)))
    return v.value


def _free_bytes():
    import torch
    free, _total = torch.cuda.mem_get_info(0)
    return free


def _states(ctx):
    """Yields (state handle, observable) for a 16-qubit QAOA Max-Cut state and a
    14-qubit random circuit with swaps (relabelled qubits) and a mixed observable."""
    cases = [(16, W.qaoa_maxcut(16, 2, seed=8)), (14, None)]
    for n, qaoa in cases:
        st = C.c_void_p()
        L.check(L.lib.qse_state_create(ctx, n, C.byref(st)))
        try:
            if qaoa is not None:
                ops, params, _, obs_t = qaoa
                p = np.ascontiguousarray(params)
                L.check(L.lib.qse_execute(st, L.dptr(ops), len(ops), p.ctypes.data_as(L._pd), p.size,
                                          None, None, 0, None))
            else:
                ops = W.random_circuit(n, 200, 21)
                L.check(L.lib.qse_execute(st, L.dptr(ops), len(ops), None, 0, None, None, 0, None))
                obs_t = ([1 << q for q in range(n)] + [0b1011, 0b11000000111], [1.0] * n + [0.5, -0.25], 0.75)
            obs, keep = L.observable(*obs_t)
            yield st, obs
        finally:
            L.lib.qse_state_destroy(st)


def test_noalloc_two_calls_match_expectation_and_allocate_nothing():
    ctx = C.c_void_p()
    L.check(L.lib.qse_ctx_create(0, C.byref(ctx)))
    _free_bytes()   # torch's own CUDA start-up happens here, outside the measured calls
    try:
        for st, obs in _states(ctx):
            # the allocating entry point first: its value is the one to match
            want = _value(L.lib.qse_expectation, st, obs)
            # one call for the per-device set-up, then two calls in a row that
            # must neither allocate nor differ
            first = _value(L.lib.qse_expectation_noalloc, st, obs)
            L.check(L.lib.qse_ctx_synchronize(ctx))
            free0 = _free_bytes()
            got1 = _value(L.lib.qse_expectation_noalloc, st, obs)
            got2 = _value(L.lib.qse_expectation_noalloc, st, obs)
            L.check(L.lib.qse_ctx_synchronize(ctx))
            free1 = _free_bytes()
            tol = 1e-12 * max(1.0, abs(want))
            for got in (first, got1, got2):
                assert abs(got - want) <= tol, (got, want)
            assert got1 == got2, (got1, got2)   # same array, same order: the same bits
            assert free1 == free0, f"device free memory changed by {free0 - free1} bytes"
    finally:
        L.lib.qse_ctx_destroy(ctx)


def test_noalloc_rejects_oversized_observable():
    ctx = C.c_void_p()
    L.check(L.lib.qse_ctx_create(0, C.byref(ctx)))
    st = C.c_void_p()
    L.check(L.lib.qse_state_create(ctx, 4, C.byref(st)))
    try:
        obs, keep = L.observable([1] * 2049, [1.0] * 2049)
        v = C.c_double()
        assert L.lib.qse_expectation_noalloc(st, C.byref(obs), C.byref(v)) == 5  # QSE_ERR_SIZE
        # the call that was refused left the entry point usable
        obs, keep = L.observable([1] * 2048, [1.0] * 2048)
        L.check(L.lib.qse_expectation_noalloc(st, C.byref(obs), C.byref(v)))
        assert abs(v.value - 2048.0) <= 1e-9   # |0000>: every Z_0 term is +1
    finally:
        L.lib.qse_state_destroy(st)
        L.lib.qse_ctx_destroy(ctx)
