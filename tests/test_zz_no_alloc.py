"""qse_expectation_noalloc: the allocation-free expectation value.

For callers that cannot allocate when they ask for <psi|O|psi> (a locked or
exhausted allocator, an embedding that forbids allocation after start-up),
the library offers an entry point whose scratch is a fixed device array
compiled into the library.  This file checks, through the C ABI, that it gives
the same value as qse_expectation on two calls in a row.  It sorts last so a
run that stops at the first failure has already run every other test, and it
passes both in a fresh process and after the other tests (the first call on
the device does the one-time address lookup either way).
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


def test_noalloc_matches_expectation_two_calls():
    ctx = C.c_void_p()
    L.check(L.lib.qse_ctx_create(0, C.byref(ctx)))
    try:
        cases = [
            # Max-Cut cost on a 16-qubit QAOA state
            (16, W.qaoa_maxcut(16, 2, seed=8)),
            # sum_i Z_i plus a few longer strings on a random 14-qubit circuit with swaps
            (14, None),
        ]
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
                want = _value(L.lib.qse_expectation, st, obs)
                got = _value(L.lib.qse_expectation_noalloc, st, obs)
                assert abs(got - want) <= 1e-12 * max(1.0, abs(want)), (n, got, want)
            finally:
                L.lib.qse_state_destroy(st)
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
    finally:
        L.lib.qse_state_destroy(st)
        L.lib.qse_ctx_destroy(ctx)
