"""C ABI: the library loads on a machine without a GPU and exports every
entry point include/qse_b200.h declares; argument errors come back as
status codes (no GPU call is made)."""
import ctypes as C
import os
import re

import pytest

from quantumsimevo_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"QSE_API\s+[\w\s\*]+?\b(qse_\w+)\s*\(", src))
    return sorted(names)


def test_header_declares_entry_points():
    assert len(_declared()) >= 45


@pytest.mark.parametrize("name", _declared())
def test_symbol_exported(name):
    assert hasattr(L.lib, name)


def test_version_and_null_handling():
    assert b"sm_100a" in L.lib.qse_version()
    assert L.lib.qse_ctx_create(0, None) == 1  # QSE_ERR_INVALID before touching the GPU
    assert b"null" in L.lib.qse_last_error()
    assert L.lib.qse_state_download(None, None) == 1
    assert L.lib.qse_ctx_destroy(None) == 0


def test_plan_describe_rejects_bad_qubits():
    ops = L.as_ops([L.make_op(L.H, 5)])
    buf = C.create_string_buffer(4096)
    need = C.c_size_t()
    rc = L.lib.qse_plan_describe(4, L.dptr(ops), 1, None, 0, 0, 0, buf, 4096, C.byref(need))
    assert rc == 2  # QSE_ERR_QUBIT
    ops = L.as_ops([L.make_op(L.MEASURE, 0)])
    assert L.lib.qse_plan_describe(4, L.dptr(ops), 1, None, 0, 0, 0, buf, 4096, C.byref(need)) == 6
