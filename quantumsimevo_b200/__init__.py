"""quantumsimevo_b200: B200 (sm_100a) state-vector backend with the interface of
SolitudeEK/QuantumSimEvo.

The compute path is libqse_b200.so (CUDA kernels + fusion planner behind a C
ABI, include/qse_b200.h); this package is its Python binding, mirroring the
reference's pybind11 module (QSEPythonModule/QuantumSimEvoPy.cpp).

The library is loaded on first use of anything that needs it (``Circuit``,
``Device``, ``lib``, ...), not by importing the package, so the plain-data
modules (``abi``, ``workloads``, ``playground``) can be used without mapping
it.  There is no fallback: if the library is missing, that first use raises.
"""
from .abi import (CNOT, CPHASE, GATE2X2, H, IDENTITY, MCPHASE, OP_DTYPE, PHASE, RNG_INJECTED, RNG_MT19937,
                  RNG_PHILOX, RX, RY, RZ, SWAP, X, Y, Z, QseError, make_op)

_LAZY = {"Circuit": "circuit", "Device": "circuit", "Noise": "circuit", "StateVector": "circuit", "lib": "_lib"}


def __getattr__(name):
    mod = _LAZY.get(name)
    if mod is None:
        raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
    import importlib
    return getattr(importlib.import_module(f".{mod}", __name__), name)


__all__ = ["Circuit", "Device", "Noise", "StateVector", "QseError", "lib", "make_op", "OP_DTYPE",
           "IDENTITY", "X", "Y", "Z", "H", "PHASE", "RX", "RY", "RZ", "CNOT", "CPHASE", "MCPHASE", "SWAP",
           "GATE2X2", "RNG_PHILOX", "RNG_MT19937", "RNG_INJECTED"]
