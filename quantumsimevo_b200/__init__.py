"""quantumsimevo_b200: B200 (sm_100a) state-vector backend with the interface of
SolitudeEK/QuantumSimEvo.

The compute path is libqse_b200.so (CUDA kernels + fusion planner behind a C
ABI, include/qse_b200.h); this package is its Python binding, mirroring the
reference's pybind11 module (QSEPythonModule/QuantumSimEvoPy.cpp).
"""
from ._lib import (CNOT, CPHASE, GATE2X2, H, IDENTITY, MCPHASE, OP_DTYPE, PHASE, RNG_INJECTED, RNG_MT19937,
                   RNG_PHILOX, RX, RY, RZ, SWAP, X, Y, Z, QseError, lib, make_op)
from .circuit import Circuit, Device, Noise, StateVector

__all__ = ["Circuit", "Device", "Noise", "StateVector", "QseError", "lib", "make_op", "OP_DTYPE",
           "IDENTITY", "X", "Y", "Z", "H", "PHASE", "RX", "RY", "RZ", "CNOT", "CPHASE", "MCPHASE", "SWAP",
           "GATE2X2", "RNG_PHILOX", "RNG_MT19937", "RNG_INJECTED"]
