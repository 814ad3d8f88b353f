"""KIR operations on the Python side of the C ABI.

``Circuit`` mirrors the reference's ``menos::Circuit`` operation list
(include/menos/circuit.h:50-150): named gates by opcode (the reference's
``menos::Opcode`` order), explicit unitaries, measurements and noise
channels.  ``ops`` is a
list of ``(opcode, qubits, params, matrix, clbit)`` tuples; ``to_mb2_ops``
packs it into the C ABI's ``mb2_op`` array.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

OPCODES = ["x", "y", "z", "h", "s", "sdg", "t", "tdg", "sx", "sxdg", "rx", "ry", "rz", "p",
           "u", "cx", "cz", "swap", "cp", "rzz", "ccx", "unitary", "measure", "channel"]
OP = {name: i for i, name in enumerate(OPCODES)}
NUM_QUBITS = {**{i: 1 for i in range(15)}, 15: 2, 16: 2, 17: 2, 18: 2, 19: 2, 20: 3}
NUM_PARAMS = {10: 1, 11: 1, 12: 1, 13: 1, 14: 3, 18: 1, 19: 1}
MAX_OP_QUBITS = 6


class MB2Op(C.Structure):
    """``mb2_op`` (include/mb2.h)."""
    _fields_ = [("opcode", C.c_int32), ("num_qubits", C.c_uint32), ("qubits", C.c_uint32 * 6),
                ("params", C.c_double * 3), ("matrix", C.POINTER(C.c_double)),
                ("clbit", C.c_uint32), ("reserved", C.c_uint32)]


class Circuit:
    def __init__(self, num_qubits: int, num_clbits: int = 0, global_phase: float = 0.0):
        self.num_qubits = int(num_qubits)
        self.num_clbits = int(num_clbits)
        self.global_phase = float(global_phase)
        self.ops: list[tuple] = []

    def gate(self, name: str, qubits, params=()) -> "Circuit":
        oc = OP[name]
        qs = tuple(int(q) for q in qubits)
        if len(qs) != NUM_QUBITS[oc]:
            raise ValueError(f"{name} takes {NUM_QUBITS[oc]} qubits")
        ps = tuple(float(p) for p in params)
        if len(ps) != NUM_PARAMS.get(oc, 0):
            raise ValueError(f"{name} takes {NUM_PARAMS.get(oc, 0)} parameters")
        self.ops.append((oc, qs, ps, None, 0))
        return self

    def unitary(self, qubits, matrix) -> "Circuit":
        qs = tuple(int(q) for q in qubits)
        m = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128))
        if m.shape != (1 << len(qs), 1 << len(qs)) or len(qs) > MAX_OP_QUBITS:
            raise ValueError("unitary shape does not match its operands")
        self.ops.append((OP["unitary"], qs, (), m, 0))
        return self

    def channel(self, qubits, kraus) -> "Circuit":
        """A noise channel (the reference's ChannelOp, include/menos/circuit.h:
        85-88): Kraus operators as a (count, 2^k, 2^k) array, k <= 5 (the
        reference's kMaxUnitaryQubits).  Only the density-matrix path
        (DensityMatrix.apply) takes it."""
        qs = tuple(int(q) for q in qubits)
        m = np.ascontiguousarray(np.asarray(kraus, dtype=np.complex128))
        if m.ndim != 3 or m.shape[0] < 1 or m.shape[1:] != (1 << len(qs), 1 << len(qs)) or not 1 <= len(qs) <= 5:
            raise ValueError("a channel takes 1..5 qubits and Kraus operators of shape (count, 2^k, 2^k)")
        self.ops.append((OP["channel"], qs, (), m, 0))
        return self

    def measure(self, qubit: int, clbit: int, readout=None) -> "Circuit":
        """readout: the measurement's readout error, P(recorded r | true t)
        as a 2x2 array [t][r] (or its 4 entries in that order), as the
        reference's ReadoutError; the density-matrix and trajectory samplers
        record the bit through it."""
        m = None
        if readout is not None:
            m = np.ascontiguousarray(np.asarray(readout, dtype=np.float64).ravel())
            if m.size != 4 or not np.all((m >= 0.0) & (m <= 1.0)):
                raise ValueError("a readout error is 4 probabilities P(recorded r | true t) at 2t + r")
        self.ops.append((OP["measure"], (int(qubit),), (), m, int(clbit)))
        self.num_clbits = max(self.num_clbits, int(clbit) + 1)
        return self

    def __len__(self) -> int:
        return len(self.ops)

    def measure_targets(self):
        """Last-write-wins (qubit, clbit) pairs, as the reference's runtime
        resolves them before the engine sees them."""
        by_clbit = {}
        for oc, qs, _ps, _m, cl in self.ops:
            if oc == OP["measure"]:
                by_clbit[cl] = qs[0]
        return [(q, c) for c, q in sorted(by_clbit.items())]


class PackedCircuit:
    """A circuit with its operations packed once into the C ABI's mb2_op
    array: every call that takes a Circuit takes it, without converting the
    operations again (a Python loop over them, ~0.7 us an operation)."""

    def __init__(self, circ: Circuit):
        self.num_qubits = circ.num_qubits
        self.num_clbits = getattr(circ, "num_clbits", 0)
        self.global_phase = circ.global_phase
        self.ops = list(circ.ops)
        self._packed = _pack(self)

    def __len__(self) -> int:
        return len(self.ops)

    def measure_targets(self):
        return Circuit.measure_targets(self)


def to_mb2_ops(circ):
    """Returns (array of MB2Op, keep-alive list of matrix buffers)."""
    if isinstance(circ, PackedCircuit):
        return circ._packed
    return _pack(circ)


def _pack(circ):
    n = len(circ.ops)
    arr = (MB2Op * max(n, 1))()
    keep = []
    for i, (oc, qs, ps, m, cl) in enumerate(circ.ops):
        o = arr[i]
        o.opcode = oc
        o.num_qubits = len(qs)
        for j, q in enumerate(qs):
            o.qubits[j] = q
        for j, p in enumerate(ps):
            o.params[j] = p
        if m is not None:
            buf = np.ascontiguousarray(m.view(np.float64).ravel())
            keep.append(buf)
            o.matrix = buf.ctypes.data_as(C.POINTER(C.c_double))
            if oc == OP["channel"]:
                o.reserved = m.shape[0]
        o.clbit = cl
    return arr, keep
