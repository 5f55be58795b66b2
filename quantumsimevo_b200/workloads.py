"""Seed-generated circuits for the five benchmark / parity configurations.

All randomness comes from ``SplitMix64`` (Steele, Lea, Flood, "Fast
splittable pseudorandom number generators", OOPSLA 2014), so the same seed
gives the same circuit in every process.  Angles are ``u * 2*pi`` (``u * pi``
for the QAOA initial parameters) with ``u`` a 53-bit uniform.

Shapes follow the reference's own circuit builders where one exists:
``qft_ops`` is ``QFT::createQFT`` (QSEplayground/QFT.cpp:9-22), and the QAOA
layer follows QSEplayground/QAOA.cpp:121-139 with the ZZ interaction written
as RZ_u(2g) RZ_v(2g) CPHASE_uv(-4g) = e^{-i g} e^{-i g Z_u Z_v} (the
reference's CNOT.RZ(4g).CNOT is e^{-i 2g Z_u Z_v}: its gamma is half of ours).
"""
from __future__ import annotations

import math

import numpy as np

from .abi import (CNOT, CPHASE, GATE2X2, H, MCPHASE, OP_DTYPE, PHASE, RX, RY, RZ, SWAP, X, Y, Z)

MASK64 = (1 << 64) - 1
TWO_PI = 2.0 * math.pi


class SplitMix64:
    def __init__(self, seed: int):
        self.state = seed & MASK64

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next_u64() >> 11) * (1.0 / 9007199254740992.0)

    def below(self, n: int) -> int:
        return int(self.uniform() * n)

    def uniforms(self, n: int) -> np.ndarray:
        return np.array([self.uniform() for _ in range(n)], dtype=np.float64)

    def permutation(self, n: int) -> list:
        p = list(range(n))
        for i in range(n - 1, 0, -1):
            j = self.below(i + 1)
            p[i], p[j] = p[j], p[i]
        return p


def _op(t, target=0, control=0, theta=0.0, controls=0, param=-1, coeff=1.0):
    return (t, target, control, param, controls, theta, coeff, (0.0,) * 8)


def to_array(ops) -> np.ndarray:
    arr = np.zeros(len(ops), dtype=OP_DTYPE)
    for i, o in enumerate(ops):
        arr[i] = o
    return arr


def layered_rotations(n=16, layers=20, seed=1):
    """Config: per layer RX, RY, RZ on every qubit (angles U[0, 2pi)), then
    CNOT(q, q+1) for even q, then for odd q.  16 qubits x 20 layers = 1260 gates."""
    rng = SplitMix64(seed)
    ops = []
    for _ in range(layers):
        for q in range(n):
            ops.append(_op(RX, q, theta=rng.uniform() * TWO_PI))
            ops.append(_op(RY, q, theta=rng.uniform() * TWO_PI))
            ops.append(_op(RZ, q, theta=rng.uniform() * TWO_PI))
        for q in range(0, n - 1, 2):
            ops.append(_op(CNOT, q + 1, q))
        for q in range(1, n - 1, 2):
            ops.append(_op(CNOT, q + 1, q))
    return to_array(ops)


def qft_ops(n, qubits=None):
    """QFT::createQFT (QFT.cpp:9-22): H(i), cphase(pi/2^(j-i), control j, target i), then swaps."""
    qs = list(range(n)) if qubits is None else list(qubits)
    m = len(qs)
    ops = []
    for i in range(m):
        ops.append(_op(H, qs[i]))
        for j in range(i + 1, m):
            ops.append(_op(CPHASE, qs[i], qs[j], math.pi / math.pow(2.0, j - i)))
    for i in range(m // 2):
        ops.append(_op(SWAP, qs[i], qs[m - 1 - i]))
    return ops


def hrz_qft(n=30, seed=2):
    """Config: H on all qubits, RZ(theta_q ~ U[0, 2pi)), then a full QFT.  30 qubits: 540 gates."""
    rng = SplitMix64(seed)
    ops = [_op(H, q) for q in range(n)]
    ops += [_op(RZ, q, theta=rng.uniform() * TWO_PI) for q in range(n)]
    ops += qft_ops(n)
    return to_array(ops)


NOISY_1Q = (H, X, Y, Z, RX, RY, RZ, PHASE)


def random_layers(n=32, layers=40, seed=3):
    """Config: per layer one uniformly chosen gate of {H, X, Y, Z, RX, RY, RZ, PHASE}
    per qubit (angles U[0, 2pi)), 16 random disjoint pairs each one of
    {CNOT, CPHASE, SWAP}, and one MCPHASE with 3 random controls on a random
    target (all four distinct).  32 qubits x 40 layers = 1960 gates."""
    rng = SplitMix64(seed)
    ops = []
    for _ in range(layers):
        for q in range(n):
            t = NOISY_1Q[rng.below(len(NOISY_1Q))]
            th = rng.uniform() * TWO_PI if t in (RX, RY, RZ, PHASE) else 0.0
            ops.append(_op(t, q, theta=th))
        perm = rng.permutation(n)
        for k in range(n // 2):
            a, b = perm[2 * k], perm[2 * k + 1]
            kind = (CNOT, CPHASE, SWAP)[rng.below(3)]
            if kind == CNOT:
                ops.append(_op(CNOT, b, a))
            elif kind == CPHASE:
                ops.append(_op(CPHASE, b, a, rng.uniform() * TWO_PI))
            else:
                ops.append(_op(SWAP, a, b))
        pick = rng.permutation(n)[:4]
        mask = (1 << pick[0]) | (1 << pick[1]) | (1 << pick[2])
        ops.append(_op(MCPHASE, pick[3], theta=rng.uniform() * TWO_PI, controls=mask))
    return to_array(ops)


def noise_rates(p=1e-3):
    """Every type of the reference's error-rate map (Noise.cpp:10-18) at rate p."""
    return {t: p for t in (X, Y, Z, H, CNOT, PHASE, RX, RY, RZ)}


def random_3_regular(n=24, seed=4, max_tries=10000):
    """Pairing-model random 3-regular graph (rejects loops and multi-edges)."""
    rng = SplitMix64(seed)
    for _ in range(max_tries):
        stubs = [v for v in range(n) for _ in range(3)]
        perm = rng.permutation(len(stubs))
        edges = set()
        ok = True
        for k in range(0, len(perm), 2):
            u, v = stubs[perm[k]], stubs[perm[k + 1]]
            if u == v or (min(u, v), max(u, v)) in edges:
                ok = False
                break
            edges.add((min(u, v), max(u, v)))
        if ok:
            return sorted(edges)
    raise RuntimeError("no simple 3-regular graph found")


def qaoa_maxcut(n=24, p=8, seed=4):
    """Config: QAOA Max-Cut on a random 3-regular graph, p layers.
    Returns (ops, params0, edges, (zmasks, weights, constant)).
    Parameters: gamma_l = params[l], beta_l = params[p + l], initial U[0, pi).
    Cost C = sum_edges (1 - Z_u Z_v)/2."""
    edges = random_3_regular(n, seed)
    rng = SplitMix64(seed ^ 0x5EED)
    params0 = np.array([rng.uniform() * math.pi for _ in range(2 * p)], dtype=np.float64)
    ops = [_op(H, q) for q in range(n)]
    for layer in range(p):
        for (u, v) in edges:
            ops.append(_op(RZ, u, param=layer, coeff=2.0))
            ops.append(_op(RZ, v, param=layer, coeff=2.0))
            ops.append(_op(CPHASE, v, u, param=layer, coeff=-4.0))
        for q in range(n):
            ops.append(_op(RX, q, param=p + layer, coeff=2.0))
    zm = [(1 << u) | (1 << v) for (u, v) in edges]
    w = [-0.5] * len(edges)
    return to_array(ops), params0, edges, (zm, w, 0.5 * len(edges))


def hea_batch(count=512, wmin=10, wmax=22, dmin=4, dmax=12, seed=5):
    """Config: `count` circuits, width U{wmin..wmax}, depth U{dmin..dmax} layers of
    [RY(q), RZ(q) on every qubit, then CNOT ring (q -> q+1 mod w)], one parameter
    per rotation (U[0, 2pi)), observable sum_i Z_i.
    Returns a list of (nqubits, ops, params, (zmasks, weights, constant))."""
    rng = SplitMix64(seed)
    out = []
    for _ in range(count):
        w = wmin + rng.below(wmax - wmin + 1)
        d = dmin + rng.below(dmax - dmin + 1)
        ops = []
        k = 0
        for _layer in range(d):
            for q in range(w):
                ops.append(_op(RY, q, param=k, coeff=1.0))
                ops.append(_op(RZ, q, param=k + 1, coeff=1.0))
                k += 2
            for q in range(w):
                ops.append(_op(CNOT, (q + 1) % w, q))
        params = np.array([rng.uniform() * TWO_PI for _ in range(k)], dtype=np.float64)
        obs = ([1 << q for q in range(w)], [1.0] * w, 0.0)
        out.append((w, to_array(ops), params, obs))
    return out


def gate2x2_unitary(rng: SplitMix64):
    """A random 2x2 unitary as the 8 doubles of qse_op.m (row-major re, im)."""
    a, b, c = rng.uniform() * TWO_PI, rng.uniform() * TWO_PI, rng.uniform() * TWO_PI
    t = rng.uniform() * math.pi / 2
    u00 = complex(math.cos(t)) * complex(math.cos(a), math.sin(a))
    u01 = -complex(math.sin(t)) * complex(math.cos(b), math.sin(b))
    u10 = complex(math.sin(t)) * complex(math.cos(c - b), math.sin(c - b))
    u11 = complex(math.cos(t)) * complex(math.cos(c - a), math.sin(c - a))
    return (u00.real, u00.imag, u01.real, u01.imag, u10.real, u10.imag, u11.real, u11.imag)


def random_circuit(n, ngates, seed, types=None, with_2x2=True):
    """Random mix of every gate type on every qubit position (parity sweeps)."""
    rng = SplitMix64(seed)
    kinds = list(types) if types else [H, X, Y, Z, PHASE, RX, RY, RZ, CNOT, CPHASE, MCPHASE, SWAP] + (
        [GATE2X2] if with_2x2 else [])
    arr = np.zeros(ngates, dtype=OP_DTYPE)
    for i in range(ngates):
        t = kinds[rng.below(len(kinds))]
        q = rng.below(n)
        if t in (CNOT, CPHASE, SWAP) and n < 2:
            t = H
        if t == MCPHASE and n < 3:
            t = PHASE
        if t in (CNOT, CPHASE, SWAP):
            c = rng.below(n - 1)
            c = c + 1 if c >= q else c
            arr[i] = (t, q, c, -1, 0, rng.uniform() * TWO_PI if t == CPHASE else 0.0, 1.0, (0.0,) * 8)
        elif t == MCPHASE:
            k = 1 + rng.below(min(3, n - 1))
            others = [x for x in rng.permutation(n) if x != q][:k]
            mask = 0
            for x in others:
                mask |= 1 << x
            arr[i] = (t, q, 0, -1, mask, rng.uniform() * TWO_PI, 1.0, (0.0,) * 8)
        elif t == GATE2X2:
            arr[i] = (t, q, 0, -1, 0, 0.0, 1.0, gate2x2_unitary(rng))
        else:
            th = rng.uniform() * TWO_PI if t in (PHASE, RX, RY, RZ) else 0.0
            arr[i] = (t, q, 0, -1, 0, th, 1.0, (0.0,) * 8)
    return arr
