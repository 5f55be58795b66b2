"""Circuit: the reference's Python-facing ``Circuit`` (QSEPythonModule/QuantumSimEvoPy.cpp:11-40)
on the B200 backend.

Same constructor, method names, argument order and semantics as the pybind11
module: gates are queued, ``execute()`` replays the whole queue on the current
state (the queue is not cleared, Circuit.cpp:64-120), ``reset()`` restores
|0..0> and clears the queue and the noise counts (Circuit.cpp:127-133),
``measure()`` collapses, ``sample(n)`` does not.  The state lives on the GPU;
``execute`` goes through the fusion planner in one call.

Differences, all additive: ``get_state_vector()`` (the reference's C++
``getStateVector`` is not bound), optional ``uniforms=`` on ``sample`` /
``measure`` to inject the draws, a ``seed`` for reproducible draws, and noise
RNG choice (``noise_rng``).  Invalid qubit indices raise instead of writing
out of bounds.
"""
from __future__ import annotations

import math
import os
import time

import numpy as np

from . import _lib as L
from ._lib import check, lib


class Device:
    """One CUDA context (device + private stream), shared by circuits."""

    _default = {}

    def __init__(self, device: int = 0):
        h = L.C.c_void_p()
        check(lib.qse_ctx_create(int(device), L.C.byref(h)))
        self.handle = h
        self.index = device

    @classmethod
    def default(cls, device: int = 0) -> "Device":
        d = cls._default.get(device)
        if d is None:
            d = cls._default[device] = Device(device)
        return d

    def set_fusion(self, enabled: bool = True, tile_qubits: int = 0, max_gates_per_pass: int = 0) -> None:
        check(lib.qse_ctx_set_fusion(self.handle, 1 if enabled else 0, int(tile_qubits), int(max_gates_per_pass)))

    def synchronize(self) -> None:
        check(lib.qse_ctx_synchronize(self.handle))

    @property
    def kernel_launches(self) -> int:
        return int(lib.qse_ctx_kernel_launches(self.handle))

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            lib.qse_ctx_destroy(h)
            self.handle = None


class StateVector:
    """Device-resident 2^n complex128 amplitudes (StateVector.h:17-44)."""

    def __init__(self, num_qubits: int, device: Device | None = None):
        self.device = device or Device.default()
        h = L.C.c_void_p()
        check(lib.qse_state_create(self.device.handle, int(num_qubits), L.C.byref(h)))
        self.handle = h
        self.num_qubits = int(num_qubits)

    @property
    def size(self) -> int:
        return 1 << self.num_qubits

    def reset(self) -> None:
        check(lib.qse_state_reset(self.handle))

    def upload(self, amplitudes) -> None:
        a = np.ascontiguousarray(np.asarray(amplitudes, dtype=np.complex128))
        if a.shape != (self.size,):
            raise ValueError(f"expected {self.size} amplitudes")
        check(lib.qse_state_upload(self.handle, L.dptr(a)))

    def download(self, first: int = 0, count: int | None = None) -> np.ndarray:
        count = self.size - first if count is None else count
        out = np.empty(count, dtype=np.complex128)
        check(lib.qse_state_download_range(self.handle, int(first), int(count), L.dptr(out)))
        return out

    def measure_qubit(self, qubit: int, u: float | None = None) -> int:
        """StateVector::measureQubit (StateVector.cpp:158-185): collapse one qubit,
        return 0 or 1.  u: the uniform draw (default: numpy's generator)."""
        u = float(np.random.random()) if u is None else float(u)
        o = L.C.c_int32()
        check(lib.qse_measure_qubit(self.handle, int(qubit), u, L.C.byref(o), None))
        return int(o.value)

    def reset_qubit(self, qubit: int, u: float | None = None) -> None:
        """StateVector::resetQubit (StateVector.cpp:187-221): measure, leave the qubit in |0>."""
        u = float(np.random.random()) if u is None else float(u)
        check(lib.qse_reset_qubit(self.handle, int(qubit), u, None, None))

    def qubit_map(self) -> list:
        m = (L.C.c_uint32 * self.num_qubits)()
        check(lib.qse_state_qubit_map(self.handle, m))
        return list(m)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            lib.qse_state_destroy(h)
            self.handle = None


class Noise:
    """Noise(N, seed=42, multiplier=1) (Noise.cpp:3-19) with device-side decisions."""

    def __init__(self, num_qubits: int, seed: int = 42, multiplier: float = 1.0, rng: int = L.RNG_PHILOX,
                 rates: dict | None = None, device: Device | None = None):
        self.device = device or Device.default()
        cfg = L.default_noise_config(True, rng, seed, multiplier, rates)
        h = L.C.c_void_p()
        check(lib.qse_noise_create(self.device.handle, int(num_qubits), L.C.byref(cfg), L.C.byref(h)))
        self.handle = h
        self.num_qubits = num_qubits
        self.rng = rng

    def reset_stats(self) -> None:
        check(lib.qse_noise_reset_stats(self.handle))

    def counts(self):
        b = (L.C.c_int32 * self.num_qubits)()
        p = (L.C.c_int32 * self.num_qubits)()
        check(lib.qse_noise_counts(self.handle, b, p))
        return list(b), list(p)

    def total_bit_flips(self) -> int:
        return sum(self.counts()[0])

    def total_phase_flips(self) -> int:
        return sum(self.counts()[1])

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            lib.qse_noise_destroy(h)
            self.handle = None


class Circuit:
    """``QuantumSimEvo.Circuit(num_qubits, simulate_pauli_noise=False)``."""

    def __init__(self, num_qubits: int, simulate_pauli_noise: bool = False, *, device: Device | None = None,
                 seed: int | None = None, noise_rng: int = L.RNG_PHILOX, noise_seed: int = 42):
        self.num_qubits = int(num_qubits)
        self.device = device or Device.default()
        self.state = StateVector(self.num_qubits, self.device)
        self.simulate_noise = bool(simulate_pauli_noise)
        self.noise = Noise(self.num_qubits, noise_seed, 1.0, noise_rng, device=self.device) if self.simulate_noise \
            else None
        self._ops = []
        self._desc = []
        self._seed = int.from_bytes(os.urandom(8), "little") if seed is None else int(seed)
        self._draws = 0
        self.last_stats = None

    # ---- gate builders (Circuit.cpp:9-62) ----
    def _q(self, q) -> int:
        q = int(q)
        if q < 0 or q >= self.num_qubits:
            raise IndexError(f"qubit {q} out of range for {self.num_qubits} qubits")
        return q

    def _push(self, op, desc):
        self._ops.append(op)
        self._desc.append(desc)

    def hadamard(self, q):
        self._push(L.make_op(L.H, self._q(q)), f"Hadamard on qubit {q}")

    def pauli_x(self, q):
        self._push(L.make_op(L.X, self._q(q)), f"PauliX on qubit {q}")

    def pauli_y(self, q):
        self._push(L.make_op(L.Y, self._q(q)), f"PauliY on qubit {q}")

    def pauli_z(self, q):
        self._push(L.make_op(L.Z, self._q(q)), f"PauliZ on qubit {q}")

    # Parameterised angles (no counterpart in the reference's pybind module,
    # QuantumSimEvoPy.cpp:11-40): with param=k the gate's angle is
    # theta + coeff * params[k], params given to execute() / gradient().
    def phase(self, theta, q, param: int = -1, coeff: float = 1.0):
        self._push(L.make_op(L.PHASE, self._q(q), theta=float(theta), param=int(param), coeff=float(coeff)),
                   f"Phase shift on qubit {q}")

    def rotate_x(self, theta, q, param: int = -1, coeff: float = 1.0):
        self._push(L.make_op(L.RX, self._q(q), theta=float(theta), param=int(param), coeff=float(coeff)),
                   f"RX on qubit {q}")

    def rotate_y(self, theta, q, param: int = -1, coeff: float = 1.0):
        self._push(L.make_op(L.RY, self._q(q), theta=float(theta), param=int(param), coeff=float(coeff)),
                   f"RY on qubit {q}")

    def rotate_z(self, theta, q, param: int = -1, coeff: float = 1.0):
        self._push(L.make_op(L.RZ, self._q(q), theta=float(theta), param=int(param), coeff=float(coeff)),
                   f"RZ on qubit {q}")

    def cnot(self, control, target):
        self._push(L.make_op(L.CNOT, self._q(target), self._q(control)),
                   f"CNOT (control: {control}, target: {target})")

    def cphase(self, theta, control, target, param: int = -1, coeff: float = 1.0):
        self._push(L.make_op(L.CPHASE, self._q(target), self._q(control), float(theta), param=int(param),
                             coeff=float(coeff)),
                   f"CPhase (theta: {theta}, control: {control}, target: {target})")

    def mcphase(self, theta, controls, target, param: int = -1, coeff: float = 1.0):
        ctl = [self._q(c) for c in controls]
        self._push(L.make_op(L.MCPHASE, self._q(target), 0, float(theta), controls=ctl, param=int(param),
                             coeff=float(coeff)),
                   f"MCPhase (theta: {theta}, target: {target}, controls: {' '.join(map(str, ctl))})")

    def swap(self, q0, q1):
        self._push(L.make_op(L.SWAP, self._q(q0), self._q(q1)), f"SWAP (q0: {q0}, q1: {q1})")

    def add_ops(self, ops) -> None:
        """Queue an OP_DTYPE array (or op tuples) at once.  The array is kept as one
        entry of the queue (no per-gate Python objects, so long circuits queue fast)."""
        arr = L.as_ops(ops).copy()
        if len(arr):
            self._ops.append(arr)
            self._desc.append(arr)

    @property
    def ops(self) -> np.ndarray:
        parts, run = [], []
        for o in self._ops:
            if isinstance(o, np.ndarray):
                if run:
                    parts.append(L.as_ops(run))
                    run = []
                parts.append(o)
            else:
                run.append(o)
        if run:
            parts.append(L.as_ops(run))
        if not parts:
            return L.as_ops([])
        return parts[0] if len(parts) == 1 else np.concatenate(parts)

    def _descriptions(self):
        for d in self._desc:
            if isinstance(d, np.ndarray):
                for o in d:
                    yield L.GATE_NAMES.get(int(o["type"]), "?")
            else:
                yield d

    # ---- execution & measurement ----
    def execute(self, print_steps: bool = False, noise_uniforms=None, params=None):
        """Replay the queue (Circuit.cpp:64-120).  With noise, the draws for each
        gate in the rate map come from the noise RNG, or from ``noise_uniforms``
        (two per noisy gate) when the noise RNG is ``RNG_INJECTED``.  params:
        values of the parameters that queued gates reference (param=k)."""
        if print_steps:
            print("Initial state: |0...0>")
            for d in self._descriptions():
                print("Executing:", d)
        ops = self.ops
        stats = L.QseExecStats()
        inj = None
        ninj = 0
        if noise_uniforms is not None:
            inj = np.ascontiguousarray(np.asarray(noise_uniforms, dtype=np.float64))
            ninj = inj.size
        t0 = time.perf_counter()
        p = None if params is None else np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
        check(lib.qse_execute(self.state.handle, L.dptr(ops) if len(ops) else None, len(ops),
                              p.ctypes.data_as(L._pd) if p is not None else None, 0 if p is None else p.size,
                              self.noise.handle if self.noise else None,
                              inj.ctypes.data_as(L._pd) if inj is not None else None, ninj, L.C.byref(stats)))
        self.last_stats = stats
        if print_steps:
            self.device.synchronize()
            ms = (time.perf_counter() - t0) * 1e3
            print(f"Executed {stats.gates} gates in {stats.passes} passes ({stats.kernels} kernels): {ms:.3f} ms (GPU)")
            if self.noise:
                print(f"Total of occured errors: \n BitFlips:{self.noise.total_bit_flips()} times\n"
                      f" PhaseFlips:{self.noise.total_phase_flips()} times.")

    def _uniforms(self, n, uniforms):
        if uniforms is not None:
            u = np.ascontiguousarray(np.asarray(uniforms, dtype=np.float64).reshape(-1))
            if u.size != n:
                raise ValueError("need one uniform per shot")
            return u
        return None

    def sample(self, num_shots, uniforms=None):
        """StateVector::sample (StateVector.cpp:77-116): outcome indices, state kept."""
        n = int(num_shots)
        out = np.empty(max(n, 0), dtype=np.uint64)
        if n <= 0:
            return []
        u = self._uniforms(n, uniforms)
        seed = (self._seed + self._draws) & ((1 << 64) - 1)
        self._draws += 0x9E3779B97F4A7C15
        check(lib.qse_sample(self.state.handle, u.ctypes.data_as(L._pd) if u is not None else None, n, seed,
                             out.ctypes.data_as(L._pu64)))
        return out

    def measure(self, uniform=None):
        """StateVector::measure (StateVector.cpp:118-156): outcome, then collapse."""
        if uniform is None:
            u1 = L.C.c_double()
            # one Philox-style draw from the circuit's seed stream
            rng = np.random.Generator(np.random.Philox(key=(self._seed + self._draws) & ((1 << 64) - 1)))
            self._draws += 1
            uniform = float(rng.random())
            del u1
        out = L.C.c_uint64()
        check(lib.qse_measure(self.state.handle, float(uniform), L.C.byref(out)))
        return int(out.value)

    def reset(self):
        self.state.reset()
        if self.noise:
            self.noise.reset_stats()
        self._ops.clear()
        self._desc.clear()

    def measure_qubit(self, q, uniform=None) -> int:
        """StateVector::measureQubit: collapse one qubit, return 0 or 1."""
        return self.state.measure_qubit(self._q(q), uniform)

    def reset_qubit(self, q, uniform=None) -> None:
        """StateVector::resetQubit: measure one qubit and leave it in |0>."""
        self.state.reset_qubit(self._q(q), uniform)

    # ---- observables and gradients (no counterpart in the reference) ----
    def expectation(self, zmasks, weights, constant: float = 0.0) -> float:
        """<psi|O|psi> of the current state for O = constant + sum_t weights[t] Z-string(zmasks[t])
        (zmask bit q = a Z on qubit q)."""
        obs, keep = L.observable(zmasks, weights, constant)
        v = L.C.c_double()
        check(lib.qse_expectation(self.state.handle, L.C.byref(obs), L.C.byref(v)))
        return v.value

    def gradient(self, params, zmasks, weights, constant: float = 0.0):
        """Runs the queued gates from |0..0> with ``params`` and returns
        (<O>, d<O>/d params) by the adjoint sweep (one forward and one reverse
        sweep over the state, whatever the number of parameters)."""
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
        obs, keep = L.observable(zmasks, weights, constant)
        ops = self.ops
        v = L.C.c_double()
        g = np.zeros(max(1, p.size))
        check(lib.qse_adjoint(self.state.handle, L.dptr(ops) if len(ops) else None, len(ops),
                              p.ctypes.data_as(L._pd), p.size, L.C.byref(obs), L.C.byref(v),
                              g.ctypes.data_as(L._pd)))
        return v.value, g[: p.size]

    # ---- utilities ----
    def get_state_vector(self) -> np.ndarray:
        return self.state.download()

    def total_probability(self) -> float:
        t = L.C.c_double()
        check(lib.qse_total_probability(self.state.handle, L.C.byref(t)))
        return t.value

    def print_state(self):
        """StateVector::printState (StateVector.cpp:250-260)."""
        n = self.num_qubits
        limit = 32 if n > 10 else (1 << n)
        amps = self.state.download(0, min(limit, 1 << n))
        for i, a in enumerate(amps):
            if abs(a) > 1e-10:
                print(f"|{format(i, 'b').zfill(n)}> : ({a.real},{a.imag})")
        if n > 10:
            print("... (truncated for large N)")
