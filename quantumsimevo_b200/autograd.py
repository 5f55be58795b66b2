"""PyTorch autograd for parameterised circuits (adjoint differentiation on the GPU).

``QuantumExpectation`` is a ``torch.autograd.Function``: its forward runs the
circuit and the adjoint sweep in one C-ABI call (``qse_adjoint``) and keeps the
gradient; its backward scales that gradient by the incoming gradient.  Gates
take their angle as ``theta + coeff * params[param]`` (``param >= 0``), so one
parameter may drive several gates (QAOA's gamma drives every ZZ term of a layer).

The observable is a weighted sum of Z-strings, O(x) = c + sum_t w_t (-1)^popc(x & z_t).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib as L
from .circuit import Device, StateVector


class ParametrizedCircuit:
    """An n-qubit gate list with parameter bindings and a diagonal observable."""

    def __init__(self, num_qubits: int, ops, zmasks, weights, constant: float = 0.0,
                 device: Device | None = None):
        self.num_qubits = int(num_qubits)
        self.ops = L.as_ops(ops)
        self.nparams = int(self.ops["param"].max()) + 1 if len(self.ops) and self.ops["param"].max() >= 0 else 0
        self.device = device or Device.default()
        self.state = StateVector(self.num_qubits, self.device)
        self._obs, self._keep = L.observable(zmasks, weights, constant)

    def value_and_grad(self, params) -> tuple[float, np.ndarray]:
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
        if p.size < self.nparams:
            raise ValueError(f"need {self.nparams} parameters, got {p.size}")
        g = np.zeros(p.size, dtype=np.float64)
        v = C.c_double()
        L.check(L.lib.qse_adjoint(self.state.handle, L.dptr(self.ops), len(self.ops), p.ctypes.data_as(L._pd),
                                  p.size, C.byref(self._obs), C.byref(v), g.ctypes.data_as(L._pd)))
        return v.value, g

    def value(self, params) -> float:
        p = np.ascontiguousarray(np.asarray(params, dtype=np.float64).reshape(-1))
        L.check(L.lib.qse_state_reset(self.state.handle))
        L.check(L.lib.qse_execute(self.state.handle, L.dptr(self.ops), len(self.ops), p.ctypes.data_as(L._pd),
                                  p.size, None, None, 0, None))
        v = C.c_double()
        L.check(L.lib.qse_expectation(self.state.handle, C.byref(self._obs), C.byref(v)))
        return v.value

    def expectation(self, params: torch.Tensor) -> torch.Tensor:
        return QuantumExpectation.apply(params, self)


class QuantumExpectation(torch.autograd.Function):
    """<psi(params)|O|psi(params)> with the adjoint gradient."""

    @staticmethod
    def forward(ctx, params: torch.Tensor, circuit: ParametrizedCircuit):
        host = params.detach().to("cpu", torch.float64).numpy()
        if params.requires_grad:
            value, grad = circuit.value_and_grad(host)
            ctx.save_for_backward(torch.as_tensor(grad, dtype=params.dtype, device=params.device))
        else:
            value = circuit.value(host)
        return torch.tensor(value, dtype=params.dtype, device=params.device)

    @staticmethod
    def backward(ctx, grad_out: torch.Tensor):
        (g,) = ctx.saved_tensors
        return grad_out * g, None


class QuantumLayer(torch.nn.Module):
    """A module holding the circuit parameters; forward() returns the expectation."""

    def __init__(self, circuit: ParametrizedCircuit, init=None):
        super().__init__()
        self.circuit = circuit
        p0 = torch.zeros(circuit.nparams, dtype=torch.float64) if init is None else torch.as_tensor(
            init, dtype=torch.float64)
        self.params = torch.nn.Parameter(p0.clone())

    def forward(self) -> torch.Tensor:
        return self.circuit.expectation(self.params)
