"""The oracle against the reference's own known answers (CPU only)."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import oracle_ffi as O
from quantumsimevo_b200 import _lib as L
from quantumsimevo_b200 import workloads as W

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _kats():
    with open(os.path.join(GOLD, "kat_qsetests.json")) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("case", _kats(), ids=lambda c: c["name"])
def test_qsetests_kat(case):
    ops = W.to_array([tuple(o) + (1.0, (0.0,) * 8) for o in case["ops"]])
    st = O.run(case["n"], ops)
    want = np.array([complex(a, b) for a, b in case["expected"]])
    # QSETests.cpp:40 compares real and imaginary parts separately at 1e-12
    assert np.all(np.abs(st.real - want.real) <= case["tolerance"])
    assert np.all(np.abs(st.imag - want.imag) <= case["tolerance"])


def test_mt19937_known_answer():
    # C++ [rand.predef]: the 10000th output of a default-constructed mt19937 is 4123659995
    g = (C.c_uint32 * 626)()
    O.oracle.orc_mt_seed(g, 5489)
    v = 0
    for _ in range(10000):
        v = O.oracle.orc_mt_next(g)
    assert v == 4123659995


def test_mt19937_canonical_matches_std_uniform_real():
    # the draw sequence Noise.cpp consumes: uniform_real_distribution<double>(0,1) over mt19937(42)
    want = np.load(os.path.join(GOLD, "ref_noise.npz"))["mt42_uniforms"]
    g = (C.c_uint32 * 626)()
    O.oracle.orc_mt_seed(g, 42)
    got = np.array([O.oracle.orc_mt_canonical(g) for _ in range(want.size)])
    assert np.array_equal(got, want)


@pytest.mark.parametrize("ctr,key,want", [
    # Random123 known-answer vectors for philox4x32-10
    ((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
    ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
    ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
     (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1)),
])
def test_philox_known_answers(ctr, key, want):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    out = (C.c_uint32 * 4)()
    O.oracle.orc_philox4x32_10(c, k, out)
    assert tuple(out) == want
