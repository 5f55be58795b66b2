"""Generates the committed golden fixtures of tests/golden/.

Run from the repository root, in a checkout where the reference sources were
compiled into oracle/_ref (``make -C oracle ref``):

    python tests/golden/make_golden.py

Outputs
  kat_qsetests.json   the known-answer vectors of QSETests/QSETests.cpp
                      (single-qubit cases :76-118, swap cases :133-149),
                      each re-run through the compiled reference to confirm it.
  ref_circuits.npz    final states of seeded random circuits over every gate
                      type and qubit position, computed by the reference's own
                      scalar backend (CircuitUnitaryOperation.cpp) via its
                      Circuit class.
  ref_noise.npz       Noise(N, seed=42, multiplier) run by the reference
                      (Noise.cpp) over a seeded gate-type sequence: flip totals
                      and the state after applyPauliNoise, plus the first
                      draws of mt19937(42) through uniform_real_distribution.
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import ctypes as C  # noqa: E402

import oracle_ffi as O  # noqa: E402
from quantumsimevo_b200 import _lib as L  # noqa: E402
from quantumsimevo_b200 import workloads as W  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
PI = 3.14159265358979323846  # QSETests.cpp:20


def op(t, target=0, control=0, theta=0.0):
    return (t, target, control, -1, 0, theta, 1.0, (0.0,) * 8)


def kat_cases():
    s = 1.0 / math.sqrt(2.0)
    th = PI / 2.0
    cases = [
        # QSETests.cpp:74-118, Program(1): one qubit, fresh |0>
        ("Hadamard", 1, [op(L.H, 0)], [(s, 0), (s, 0)]),
        ("PauliX", 1, [op(L.X, 0)], [(0, 0), (1, 0)]),
        ("PauliY", 1, [op(L.Y, 0)], [(0, 0), (0, 1)]),
        ("PauliZ", 1, [op(L.Z, 0)], [(1, 0), (0, 0)]),
        ("Phase", 1, [op(L.PHASE, 0, theta=PI / 2.0)], [(1, 0), (0, 0)]),
        ("RotateX", 1, [op(L.RX, 0, theta=th)], [(math.cos(th / 2), 0), (0, -math.sin(th / 2))]),
        ("RotateY", 1, [op(L.RY, 0, theta=th)], [(math.cos(th / 2), 0), (math.cos(th / 2), 0)]),
        ("RotateZ", 1, [op(L.RZ, 0, theta=th)], [(math.cos(th / 2), -math.sin(th / 2)), (0, 0)]),
        # QSETests.cpp:133-149, Circuit(2), qubit 0 = LSB
        ("Swap |00> unchanged", 2, [op(L.SWAP, 0, 1)], [(1, 0), (0, 0), (0, 0), (0, 0)]),
        ("Swap |01> -> |10>", 2, [op(L.X, 0), op(L.SWAP, 0, 1)], [(0, 0), (0, 0), (1, 0), (0, 0)]),
        ("Swap |10> -> |01>", 2, [op(L.X, 1), op(L.SWAP, 0, 1)], [(0, 0), (1, 0), (0, 0), (0, 0)]),
        ("Swap H(0) superposition", 2, [op(L.H, 0), op(L.SWAP, 0, 1)], [(s, 0), (0, 0), (s, 0), (0, 0)]),
        ("Swap self-inverse", 2, [op(L.X, 0), op(L.SWAP, 0, 1), op(L.SWAP, 0, 1)],
         [(0, 0), (1, 0), (0, 0), (0, 0)]),
    ]
    return cases


def main():
    ref = O.load_reference(gpu=False)
    if ref is None:
        raise SystemExit("oracle/_ref/libqse_ref_cpu.so is missing: run `make -C oracle ref` first")
    ref.ref_set_quiet(1)

    kats = []
    for name, n, ops, exp in kat_cases():
        arr = W.to_array(ops)
        got = O.ref_run(ref, n, arr)
        want = np.array([complex(a, b) for a, b in exp])
        assert np.max(np.abs(got - want)) <= 1e-12, (name, got, want)
        kats.append({"name": name, "n": n, "ops": [list(o[:6]) for o in ops],
                     "expected": [[float(a), float(b)] for a, b in exp], "tolerance": 1e-12})
    with open(os.path.join(OUT, "kat_qsetests.json"), "w") as f:
        json.dump({"source": "QSETests/QSETests.cpp:26-50 (validate, tol 1e-12), :74-170", "cases": kats}, f,
                  indent=1)

    circuits = {}
    idx = 0
    for n in (1, 2, 3, 4, 5, 6, 8):
        for rep in range(3):
            seed = 1000 + 17 * n + rep
            arr = W.random_circuit(n, 12 * n + 8, seed)
            # the reference Circuit has no builder for a generic 2x2: keep those out
            arr = arr[arr["type"] != L.GATE2X2]
            st = O.ref_run(ref, n, arr)
            circuits[f"c{idx}_n"] = np.array(n)
            circuits[f"c{idx}_ops"] = arr
            circuits[f"c{idx}_state"] = st
            idx += 1
    circuits["count"] = np.array(idx)
    np.savez_compressed(os.path.join(OUT, "ref_circuits.npz"), **circuits)

    # Noise with seed 42 (Circuit.cpp:5) over a seeded sequence of gate types
    rng = W.SplitMix64(77)
    noise = {}
    for case, (n, ngates, mult) in enumerate(((3, 200, 20.0), (5, 400, 10.0), (6, 1000, 1.0))):
        types = np.array([[L.X, L.Y, L.Z, L.H, L.CNOT, L.PHASE, L.RX, L.RY, L.RZ, L.CPHASE, L.SWAP,
                           L.MCPHASE][rng.below(12)] for _ in range(ngates)], dtype=np.int32)
        targets = np.array([rng.below(n) for _ in range(ngates)], dtype=np.uint32)
        st0 = np.array([complex(rng.uniform() - 0.5, rng.uniform() - 0.5) for _ in range(1 << n)])
        st = st0.copy()
        bt, pt = C.c_uint64(), C.c_uint64()
        ref.ref_noise_run(n, 42, mult, types.ctypes.data_as(C.POINTER(C.c_int)),
                          targets.ctypes.data_as(C.POINTER(C.c_uint)), ngates, st.ctypes.data_as(C.c_void_p),
                          C.byref(bt), C.byref(pt))
        noise[f"k{case}_n"] = np.array(n)
        noise[f"k{case}_mult"] = np.array(mult)
        noise[f"k{case}_types"] = types
        noise[f"k{case}_targets"] = targets
        noise[f"k{case}_in"] = st0
        noise[f"k{case}_out"] = st
        noise[f"k{case}_bits"] = np.array(bt.value)
        noise[f"k{case}_phases"] = np.array(pt.value)
    noise["count"] = np.array(3)
    u = np.empty(2000, dtype=np.float64)
    ref.ref_std_uniforms(42, u.size, u.ctypes.data_as(C.POINTER(C.c_double)))
    noise["mt42_uniforms"] = u
    np.savez_compressed(os.path.join(OUT, "ref_noise.npz"), **noise)
    print("wrote", os.listdir(OUT))


if __name__ == "__main__":
    main()
