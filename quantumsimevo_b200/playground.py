"""Circuits of the reference's playground programs (QSEplayground/) as op
lists for ``Circuit.add_ops``, and the paper's wall-clock workloads built
from them (construct -> execute -> sample(shots)).

Each builder follows the reference function it names gate for gate, in the
same order and with the same angles, so a circuit built here and the
reference's own circuit produce the same state.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .abi import CNOT, CPHASE, H, MCPHASE, RX, RZ, SWAP, X
from .workloads import _op, to_array

PI = 3.14159265358979323846   # Grover.cpp:10, QFT.cpp:6


def ghz(n: int) -> np.ndarray:
    """ghz() (QSEplayground.cpp:134-151): H(0), then CNOT(j, j+1) for j < n-1."""
    ops = [_op(H, 0)]
    ops += [_op(CNOT, j + 1, j) for j in range(n - 1)]
    return to_array(ops)


def _qft_body(qs) -> list:
    """QFT::createQFT (QFT.cpp:9-22): H(q_i), cphase(pi/2^(j-i), control q_j, target q_i), then swaps."""
    m = len(qs)
    ops = []
    for i in range(m):
        ops.append(_op(H, qs[i]))
        for j in range(i + 1, m):
            ops.append(_op(CPHASE, qs[i], qs[j], PI / math.pow(2.0, j - i)))
    for i in range(m // 2):
        ops.append(_op(SWAP, qs[i], qs[m - 1 - i]))
    return ops


def _iqft_body(qs) -> list:
    """QFT::createIQFT (QFT.cpp:24-37): swaps, then for i = m-1..0: cphase(-pi/2^(j-i), q_j, q_i)
    for j = m-1..i+1, then H(q_i)."""
    m = len(qs)
    ops = [_op(SWAP, qs[i], qs[m - 1 - i]) for i in range(m // 2)]
    for i in range(m - 1, -1, -1):
        for j in range(m - 1, i, -1):
            ops.append(_op(CPHASE, qs[i], qs[j], -PI / math.pow(2.0, j - i)))
        ops.append(_op(H, qs[i]))
    return ops


def qft(n: int) -> np.ndarray:
    """QFT::runQFT (QFT.cpp:39-71): X(0), then the QFT over qubits 0..n-1."""
    return to_array([_op(X, 0)] + _qft_body(list(range(n))))


def iqft(n: int) -> np.ndarray:
    """QFT::runIQFT (QFT.cpp:73-105): X(0), then the inverse QFT over qubits 0..n-1."""
    return to_array([_op(X, 0)] + _iqft_body(list(range(n))))


def grover_size(target: int):
    """Grover::runGrover (Grover.cpp:12-26): the fewest qubits n with 2^n > target, and
    round(pi/4 sqrt(2^n)) iterations (std::round: halves away from zero), at least 1."""
    n = 1
    while (1 << n) <= target:
        n += 1
    it = int(math.floor((PI / 4.0) * math.sqrt(float(1 << n)) + 0.5))
    return n, max(it, 1)


def grover(target: int, iterations: int | None = None) -> np.ndarray:
    """Grover::createGroverCircuit (Grover.cpp:65-75): H on all qubits, then `iterations`
    times the oracle (Grover.cpp:77-89) and the diffusion (Grover.cpp:91-105)."""
    n, it = grover_size(target)
    if iterations is not None:
        it = iterations
    ctrl = (1 << (n - 1)) - 1          # controls 0..n-2, target n-1
    flip = [_op(X, i) for i in range(n) if not ((target >> i) & 1)]
    oracle = flip + [_op(MCPHASE, n - 1, 0, PI, ctrl)] + flip
    hs = [_op(H, i) for i in range(n)]
    xs = [_op(X, i) for i in range(n)]
    diffusion = hs + xs + [_op(MCPHASE, n - 1, 0, PI, ctrl)] + xs + hs
    return np.concatenate([to_array(hs), np.tile(to_array(oracle + diffusion), it)])


# qaoa() (QSEplayground.cpp:47-88): 30 nodes, a ring plus the chords i -- i+15, p = 3,
# gamma = pi/8 and beta = pi/3 per layer (as float), 1.5e6 shots
MAXCUT30_EDGES = [(i, (i + 1) % 30) for i in range(30)] + [(i, i + 15) for i in range(15)]


def qaoa_maxcut(n: int, edges, gamma, beta) -> np.ndarray:
    """QAOA::runQAOA (QAOA.cpp:105-144): H on all qubits; per layer i, for every edge (u, v)
    CNOT(u, v) RZ(4 gamma_i, v) CNOT(u, v), then RX(2 beta_i) on every qubit.  The angles
    are the reference's float products (4 * gamma[i] and 2 * beta[i] in single precision)."""
    ops = [_op(H, q) for q in range(n)]
    for g, b in zip(gamma, beta):
        g4 = float(np.float32(4.0) * np.float32(g))
        b2 = float(np.float32(2.0) * np.float32(b))
        for u, v in edges:
            ops += [_op(CNOT, v, u), _op(RZ, v, theta=g4), _op(CNOT, v, u)]
        ops += [_op(RX, q, theta=b2) for q in range(n)]
    return to_array(ops)


def maxcut30(p: int = 3) -> np.ndarray:
    return qaoa_maxcut(30, MAXCUT30_EDGES, [math.pi / 8] * p, [math.pi / 3] * p)


# tsp() (QSEplayground.cpp:16-45): 5 cities -> 25 qubits; TVS::runTVS(dist5, -1, 1, 0.8, 0.4, 100000)
TSP5_DIST = [[0, 3, 4, 2, 7], [3, 0, 5, 7, 6], [4, 5, 0, 6, 3], [2, 7, 6, 0, 5], [7, 6, 3, 5, 0]]


def tsp_index(city: int, step: int, n: int) -> int:
    """TVS::getIndex (TVS.cpp:10-13): qubit of "city at step"."""
    return city * n + step


def tsp_ising(n, penalty, weight, dist, row_constraint=True, col_constraint=True):
    """TVS::buildIsing (TVS.cpp:31-99): the TSP QUBO in Ising form, fields h and couplings
    J (pairs i < j), accumulated in the reference's order so every coefficient is the same
    double.  Returns (h, pairs, coeffs) with pairs in first-insertion order."""
    qubits = n * n
    h = [0.0] * qubits
    J = {}

    def add_zz(a, b, c):
        if a > b:
            a, b = b, a
        J[(a, b)] = J.get((a, b), 0.0) + c

    def add_linear(i, c):
        h[i] -= c / 2.0

    def add_quad(i, j, q):
        h[i] -= q / 4.0
        h[j] -= q / 4.0
        add_zz(i, j, q / 4.0)

    def add_constraint(group):
        for a in range(len(group)):
            add_linear(group[a], -penalty)
            for b in range(a + 1, len(group)):
                add_quad(group[a], group[b], 2.0 * penalty)

    if row_constraint:
        for v in range(n):
            add_constraint([tsp_index(v, t, n) for t in range(n)])
    if col_constraint:
        for t in range(n):
            add_constraint([tsp_index(v, t, n) for v in range(n)])
    for u in range(n):
        for v in range(n):
            if u == v:
                continue
            q = weight * dist[u][v]
            for t in range(n):
                add_quad(tsp_index(u, t, n), tsp_index(v, (t + 1) % n, n), q)
    pairs = [k for k, c in J.items() if abs(c) >= 1e-15]
    return h, pairs, [J[k] for k in pairs]


def tsp_schedule(penalty, weight, gamma, beta, layers, dist):
    """TVS::runTVS (TVS.cpp:292-308): the automatic penalty (negative -> weight * maxDist * n
    + 1) and the per-layer ramps gamma_k = gamma (k+1)/p, beta_k = beta (1 - (k+1)/p) + beta/4."""
    n = len(dist)
    if penalty < 0.0:
        penalty = weight * max(max(r) for r in dist) * float(n) + 1.0
    layers = max(layers, 1)
    gammas, betas = [], []
    for k in range(layers):
        frac = 1.0 if layers == 1 else (k + 1) / layers
        gammas.append(gamma * frac)
        betas.append(beta * (1.0 - frac) + beta * 0.25)
    return penalty, gammas, betas


def tsp_xy_qaoa(dist, penalty, weight, gammas, betas) -> np.ndarray:
    """TVS::createCircuit (TVS.cpp:118-179): X on the identity tour, then per layer the
    ZZ phases CNOT RZ(2 gamma J) CNOT and RZ(2 gamma h) on every qubit (column penalty and
    route cost; the row constraint is left to the mixer), then the XY ring mixer inside
    each city row, each pair as Rxx(2 beta) (H-conjugated CNOT RZ CNOT) then Ryy(2 beta)
    (RX(+-pi/2)-conjugated).  The reference emits the ZZ pairs in its hash map's order;
    they commute, so any fixed order gives the same state up to rounding."""
    n = len(dist)
    qubits = n * n
    h, pairs, coeffs = tsp_ising(n, penalty, weight, dist, row_constraint=False, col_constraint=True)
    ops = [_op(X, tsp_index(v, v, n)) for v in range(n)]
    for gamma, beta in zip(gammas, betas):
        for (q1, q2), c in zip(pairs, coeffs):
            ops += [_op(CNOT, q2, q1), _op(RZ, q2, theta=2 * gamma * c), _op(CNOT, q2, q1)]
        ops += [_op(RZ, q, theta=2 * gamma * h[q]) for q in range(qubits)]
        for v in range(n):
            for t in range(n):
                a, b = tsp_index(v, t, n), tsp_index(v, (t + 1) % n, n)
                ops += [_op(H, a), _op(H, b), _op(CNOT, b, a), _op(RZ, b, theta=2 * beta), _op(CNOT, b, a),
                        _op(H, a), _op(H, b),
                        _op(RX, a, theta=PI / 2), _op(RX, b, theta=PI / 2),
                        _op(CNOT, b, a), _op(RZ, b, theta=2 * beta), _op(CNOT, b, a),
                        _op(RX, a, theta=-PI / 2), _op(RX, b, theta=-PI / 2)]
    return to_array(ops)


def tsp5() -> np.ndarray:
    penalty, gammas, betas = tsp_schedule(-1.0, 1.0, 0.8, 0.4, 4, TSP5_DIST)
    return tsp_xy_qaoa(TSP5_DIST, penalty, 1.0, gammas, betas)


@dataclass
class Workload:
    name: str
    qubits: int
    shots: int
    build: object        # () -> op array
    paper_ms: float | None = None
    paper_what: str = ""


def workloads() -> list:
    """The paper's timed playground workloads (times: wall clock for construct -> execute ->
    sample; CPU rows on an i9-12900H AVX2 backend, GPU rows on an RTX 3070 Ti Laptop)."""
    gt = 29123321                        # QSEplayground.cpp:182: Grover::runGrover(29123321, 10000)
    return [
        Workload("ghz25", 25, 1000, lambda: ghz(25), 762.0, "CUDA, RTX 3070 Ti Laptop"),
        Workload("ghz28", 28, 1000, lambda: ghz(28), 5064.0, "CUDA, RTX 3070 Ti Laptop"),
        Workload("ghz30", 30, 1000, lambda: ghz(30), 29000.0, "AVX2 CPU"),
        Workload("qft25", 25, 1000, lambda: qft(25), 1053.0, "CUDA, RTX 3070 Ti Laptop"),
        Workload("qft28", 28, 1000, lambda: qft(28), 6838.0, "CUDA, RTX 3070 Ti Laptop"),
        Workload("qft30", 30, 1000, lambda: qft(30), 130000.0, "AVX2 CPU"),
        Workload("iqft25", 25, 1000, lambda: iqft(25), 1043.0, "CUDA, RTX 3070 Ti Laptop"),
        Workload("iqft28", 28, 1000, lambda: iqft(28), 6844.0, "CUDA, RTX 3070 Ti Laptop"),
        Workload("iqft30", 30, 1000, lambda: iqft(30), 125000.0, "AVX2 CPU"),
        Workload("grover25", grover_size(gt)[0], 10000, lambda: grover(gt), 4950000.0, "CUDA"),
        Workload("maxcut30_p3", 30, 1500000, lambda: maxcut30(3), 278000.0, "CPU (30 q exceeds 8 GB)"),
        Workload("tsp5_p4", 25, 100000, tsp5, 12000.0, "CUDA"),
    ]
