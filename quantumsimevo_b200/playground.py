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

from ._lib import CNOT, CPHASE, H, MCPHASE, RX, RZ, SWAP, X
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
    ]
