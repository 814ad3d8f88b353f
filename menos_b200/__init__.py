"""menos_b200 -- a B200-native (sm_100a) dense statevector engine for MENOS.

The compute path is libmenos_b200.so (C ABI: include/mb2.h), hand-written
CUDA for sm_100a with a C++ host layer.  This package is its Python face:
``engine`` (contexts, device states, the SimulationEngine mirror),
``circuit`` (KIR operations) and ``workloads`` (seeded benchmark circuits).
"""
from .circuit import OP, Circuit
from .engine import (B200DenseEngine, Context, DensityMatrix, DeviceState, EngineExecutionRequest,
                     EngineExecutionResult, PauliTerm)

__all__ = ["OP", "Circuit", "B200DenseEngine", "Context", "DensityMatrix", "DeviceState", "EngineExecutionRequest",
           "EngineExecutionResult", "PauliTerm"]
