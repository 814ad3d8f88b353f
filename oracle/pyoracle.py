"""TEST INFRASTRUCTURE: ctypes bindings of the two CPU checkers.

* ``Oracle``  -- build/liboracle.so, this repository's plain-C restatement of
  the reference MENOS CPU dense algorithm (oracle.c).
* ``RefLib``  -- _ref/libmenos_ref.so, the reference's own CPU sources
  compiled here (Makefile), reached through ref_shim.cpp.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module, and only to check or time against; the product package
never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libmenos_ref.so")
REF_CUDA_SO = os.path.join(HERE, "_ref", "libmenos_ref_cuda.so")

# Opcodes: the reference's menos::Opcode order (include/menos/circuit.h:17-41).
OPCODES = ["x", "y", "z", "h", "s", "sdg", "t", "tdg", "sx", "sxdg", "rx", "ry", "rz", "p",
           "u", "cx", "cz", "swap", "cp", "rzz", "ccx", "unitary", "measure", "channel"]
OP = {name: i for i, name in enumerate(OPCODES)}
NUM_PARAMS = {10: 1, 11: 1, 12: 1, 13: 1, 14: 3, 18: 1, 19: 1}

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build(ref: bool = True) -> None:
    """Compiles the oracle (and the reference library when its sources exist)."""
    target = "all" if ref else "oracle"
    subprocess.run(["make", "-s", "-C", HERE, target], check=True)


class Circuit:
    """A flat operation list in the C ABI's op layout (parallel arrays)."""

    def __init__(self, num_qubits: int, global_phase: float = 0.0):
        self.num_qubits = num_qubits
        self.global_phase = global_phase
        self.ops: list[tuple] = []  # (opcode, qubits, params, matrix or None, clbit)

    def gate(self, name: str, qubits, params=()):
        self.ops.append((OP[name], tuple(int(q) for q in qubits), tuple(float(p) for p in params), None, 0))
        return self

    def unitary(self, qubits, matrix):
        m = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128))
        self.ops.append((OP["unitary"], tuple(int(q) for q in qubits), (), m, 0))
        return self

    def measure(self, qubit: int, clbit: int, readout=None):
        """readout: P(recorded r | true t) at 2t + r (the reference's ReadoutError)."""
        m = None if readout is None else np.ascontiguousarray(np.asarray(readout, np.float64).ravel())
        self.ops.append((OP["measure"], (int(qubit),), (), m, int(clbit)))
        return self

    def channel(self, qubits, kraus):
        """A noise channel: Kraus operators (count, 2^k, 2^k)."""
        m = np.ascontiguousarray(np.asarray(kraus, dtype=np.complex128))
        self.ops.append((OP["channel"], tuple(int(q) for q in qubits), (), m, 0))
        return self

    def arrays(self):
        return arrays(self)


def arrays(circ):
    """Parallel arrays (opcode, nq, qubits[6], params[3], matrices) of any
    circuit-like object with an ``ops`` list of (opcode, qubits, params,
    matrix, clbit) tuples."""
    n = len(circ.ops)
    opcode = np.zeros(max(n, 1), np.int32)
    nq = np.zeros(max(n, 1), np.uint32)
    qubits = np.zeros(max(n, 1) * 6, np.uint32)
    params = np.zeros(max(n, 1) * 3, np.float64)
    mats = []
    for i, (oc, qs, ps, m, _cl) in enumerate(circ.ops):
        opcode[i] = oc
        nq[i] = len(qs)
        qubits[6 * i:6 * i + len(qs)] = qs
        params[3 * i:3 * i + len(ps)] = ps
        if m is not None and oc != OP["measure"]:  # a measurement's readout error is not a matrix here
            mats.append(m.view(np.float64).ravel())
    matrices = np.ascontiguousarray(np.concatenate(mats)) if mats else np.zeros(1, np.float64)
    return n, opcode, nq, qubits, params, matrices


class _MB2Op(C.Structure):
    _fields_ = [("opcode", C.c_int32), ("num_qubits", C.c_uint32), ("qubits", C.c_uint32 * 6),
                ("params", C.c_double * 3), ("matrix", C.POINTER(C.c_double)),
                ("clbit", C.c_uint32), ("reserved", C.c_uint32)]


def ops_struct_array(circ: Circuit):
    """The circuit as an array of ``mb2_op`` (the C ABI's struct), plus the
    matrix buffers it points into (kept alive by the caller)."""
    arr = (_MB2Op * max(len(circ.ops), 1))()
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


class Oracle:
    """The plain-C restatement (oracle.c)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(ref=False)
        L = C.CDLL(path)
        L.orc_uniforms.argtypes = [C.c_uint64, C.c_uint64, _dp]
        L.orc_words.argtypes = [C.c_uint64, C.c_uint64, _u64p]
        L.orc_gate_matrix.argtypes = [C.c_int, _dp, _dp]
        L.orc_gate_matrix.restype = C.c_int
        L.orc_apply_generic.argtypes = [_dp, C.c_uint64, _dp, _u32p, C.c_uint32]
        L.orc_initialize.argtypes = [_dp, C.c_uint64, C.c_double]
        L.orc_expectation.argtypes = [_dp, C.c_uint64, C.c_uint64, C.c_uint64, _dp]
        L.orc_sample.argtypes = [_dp, C.c_uint64, C.c_uint64, C.c_uint64, _u32p, C.c_uint32, _u64p, _u64p,
                                 C.c_uint64]
        L.orc_sample.restype = C.c_int64
        L.orc_sample_basis.argtypes = [_dp, C.c_uint64, C.c_uint64, C.c_uint64, _u64p]
        L.orc_plan_fusion.argtypes = [C.c_uint32, _i32p, _u32p, _u32p, _dp, _dp, _u32p, _u32p, _u32p, _u32p]
        L.orc_plan_fusion.restype = C.c_int64
        L.orc_run.argtypes = [C.c_uint32, C.c_uint32, _i32p, _u32p, _u32p, _dp, _dp, C.c_double, C.c_int, _dp]
        L.orc_run.restype = C.c_int
        L.orc_fused_block_matrix.argtypes = [C.c_uint32, _i32p, _u32p, _u32p, _dp, _dp, C.c_uint32, _dp]
        L.orc_fused_block_matrix.restype = C.c_int
        self.L = L

    def uniforms(self, seed: int, n: int) -> np.ndarray:
        out = np.zeros(max(n, 1), np.float64)
        self.L.orc_uniforms(seed, n, out)
        return out[:n]

    def words(self, seed: int, n: int) -> np.ndarray:
        out = np.zeros(max(n, 1), np.uint64)
        self.L.orc_words(seed, n, out)
        return out[:n]

    def gate_matrix(self, opcode: int, params=()) -> np.ndarray:
        p = np.zeros(3, np.float64)
        p[:len(params)] = params
        out = np.zeros(2 * 64, np.float64)
        dim = self.L.orc_gate_matrix(int(opcode), p, out)
        return out[:2 * dim * dim].view(np.complex128).reshape(dim, dim).copy()

    def apply_generic(self, state: np.ndarray, matrix: np.ndarray, operands) -> None:
        assert state.dtype == np.complex128 and state.flags.c_contiguous
        m = np.ascontiguousarray(np.asarray(matrix, np.complex128)).view(np.float64).ravel()
        ops = np.asarray(operands, np.uint32)
        self.L.orc_apply_generic(state.view(np.float64), state.size, m, ops, len(ops))

    def initialize(self, num_qubits: int, global_phase: float = 0.0) -> np.ndarray:
        s = np.zeros(1 << num_qubits, np.complex128)
        self.L.orc_initialize(s.view(np.float64), s.size, global_phase)
        return s

    def expectation(self, state: np.ndarray, x: int, z: int) -> complex:
        out = np.zeros(2, np.float64)
        self.L.orc_expectation(state.view(np.float64), state.size, x, z, out)
        return complex(out[0], out[1])

    def sample(self, state: np.ndarray, shots: int, seed: int, targets) -> dict:
        t = np.asarray(targets, np.uint32).ravel()
        cap = max(shots, 1)
        outc = np.zeros(cap, np.uint64)
        cnt = np.zeros(cap, np.uint64)
        d = self.L.orc_sample(state.view(np.float64), state.size, shots, seed, t, len(t) // 2, outc, cnt, cap)
        assert d >= 0
        return {int(o): int(c) for o, c in zip(outc[:d], cnt[:d])}

    def sample_basis(self, state: np.ndarray, shots: int, seed: int) -> np.ndarray:
        out = np.zeros(max(shots, 1), np.uint64)
        self.L.orc_sample_basis(state.view(np.float64), state.size, shots, seed, out)
        return out[:shots]

    def plan_fusion(self, circ: Circuit):
        n, opcode, nq, qubits, params, mats = arrays(circ)
        order = np.zeros(max(n, 1), np.uint32)
        bb = np.zeros(n + 1, np.uint32)
        bq = np.zeros(max(64 * n, 1), np.uint32)
        qb = np.zeros(n + 1, np.uint32)
        blocks = self.L.orc_plan_fusion(n, opcode, nq, qubits, params, mats, order, bb, bq, qb)
        return order[:n], bb[:blocks + 1], bq[:qb[blocks]], qb[:blocks + 1]

    def fused_block_matrix(self, circ: Circuit, block: int) -> np.ndarray:
        n, opcode, nq, qubits, params, mats = arrays(circ)
        out = np.zeros(2 * 64 * 64, np.float64)
        dim = self.L.orc_fused_block_matrix(n, opcode, nq, qubits, params, mats, block, out)
        return out[:2 * dim * dim].view(np.complex128).reshape(dim, dim).copy()

    def run(self, circ: Circuit, fuse_gates: bool = True) -> np.ndarray:
        n, opcode, nq, qubits, params, mats = arrays(circ)
        state = np.zeros(1 << circ.num_qubits, np.complex128)
        rc = self.L.orc_run(circ.num_qubits, n, opcode, nq, qubits, params, mats, circ.global_phase,
                            1 if fuse_gates else 0, state.view(np.float64))
        assert rc == 0
        return state


class RefLib:
    """The reference's own CPU dense engine (compiled from its sources)."""

    available = os.path.exists(REF_SO)

    def __init__(self, path: str = REF_SO):
        L = C.CDLL(path)
        L.ref_generate_matrix.argtypes = [C.c_int, _dp, _dp, C.c_uint32]
        L.ref_generate_matrix.restype = C.c_int
        L.ref_apply_matrix.argtypes = [_dp, C.c_uint64, _dp, _u32p, C.c_uint32, C.c_uint32]
        L.ref_apply_matrix_generic.argtypes = [_dp, C.c_uint64, _dp, _u32p, C.c_uint32, C.c_uint32]
        L.ref_expectation_of_term.argtypes = [_dp, C.c_uint64, C.c_uint64, C.c_uint64, _dp]
        L.ref_uniforms.argtypes = [C.c_uint64, C.c_uint64, _dp]
        L.ref_sample.argtypes = [_dp, C.c_uint64, C.c_uint64, C.c_uint64, _u32p, C.c_uint32, C.c_uint32,
                                 _u64p, _u64p, C.c_uint64]
        L.ref_sample.restype = C.c_int64
        L.ref_plan_fusion.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_plan_fusion.restype = C.c_int64
        L.ref_fused_block_matrix.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, _dp, C.c_uint32]
        L.ref_fused_block_matrix.restype = C.c_int
        L.ref_run_dense.argtypes = [C.c_uint32, C.c_void_p, C.c_uint32, C.c_double, C.c_int, C.c_uint32,
                                    C.c_void_p, C.c_uint64, C.c_uint64, C.c_void_p, C.c_uint32, C.c_uint32,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                    C.c_void_p, C.c_void_p]
        L.ref_run_dense.restype = C.c_int
        if hasattr(L, "ref_run_cuda"):  # the library with the reference's CUDA engine
            L.ref_run_cuda.argtypes = L.ref_run_dense.argtypes
            L.ref_run_cuda.restype = C.c_int
        L.ref_run_plan.argtypes = [C.c_uint32, C.c_void_p, C.c_uint32, C.c_double, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]
        L.ref_run_plan.restype = C.c_int
        L.ref_run_dm.argtypes = [C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64,
                                 C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
        L.ref_run_dm.restype = C.c_int
        L.ref_run_trajectories.argtypes = [C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint64, C.c_uint64, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint64,
                                           C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_run_trajectories.restype = C.c_int
        L.ref_pass_plan.argtypes = [C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p,
                                    C.c_uint64]
        L.ref_pass_plan.restype = C.c_int64
        L.ref_last_error.restype = C.c_char_p
        L.ref_default_threads.restype = C.c_uint32
        L.ref_kernel_isa.restype = C.c_int
        self.L = L

    def gate_matrix(self, opcode: int, params=()) -> np.ndarray:
        p = np.zeros(3, np.float64)
        p[:len(params)] = params
        out = np.zeros(2 * 64, np.float64)
        n = self.L.ref_generate_matrix(int(opcode), p, out, out.size)
        assert n > 0, self.L.ref_last_error()
        dim = int(round(n ** 0.5))
        return out[:2 * n].view(np.complex128).reshape(dim, dim).copy()

    def apply_matrix(self, state, matrix, operands, threads=1, generic=False):
        m = np.ascontiguousarray(np.asarray(matrix, np.complex128)).view(np.float64).ravel()
        ops = np.asarray(operands, np.uint32)
        f = self.L.ref_apply_matrix_generic if generic else self.L.ref_apply_matrix
        rc = f(state.view(np.float64), state.size, m, ops, len(ops), threads)
        assert rc == 0, self.L.ref_last_error()

    def expectation(self, state, x, z) -> complex:
        out = np.zeros(2, np.float64)
        self.L.ref_expectation_of_term(state.view(np.float64), state.size, x, z, out)
        return complex(out[0], out[1])

    def uniforms(self, seed, n):
        out = np.zeros(max(n, 1), np.float64)
        self.L.ref_uniforms(seed, n, out)
        return out[:n]

    def sample(self, state, shots, seed, targets, width=None) -> dict:
        t = np.asarray(targets, np.uint32).ravel()
        if width is None:
            width = int(max(t[1::2]) + 1) if len(t) else 0
        cap = max(shots, 1)
        outc = np.zeros(cap, np.uint64)
        cnt = np.zeros(cap, np.uint64)
        d = self.L.ref_sample(state.view(np.float64), state.size, shots, seed, t, len(t) // 2, width, outc, cnt,
                              cap)
        assert d >= 0
        return {int(o): int(c) for o, c in zip(outc[:d], cnt[:d])}

    def plan_fusion(self, circ: Circuit):
        arr, keep = ops_struct_array(circ)
        n = len(circ.ops)
        order = np.zeros(max(n, 1), np.uint32)
        bb = np.zeros(n + 1, np.uint32)
        bq = np.zeros(max(64 * n, 1), np.uint32)
        qb = np.zeros(n + 1, np.uint32)
        blocks = self.L.ref_plan_fusion(C.addressof(arr), n, order.ctypes.data, bb.ctypes.data, bq.ctypes.data,
                                        qb.ctypes.data)
        del keep
        return order[:n], bb[:blocks + 1], bq[:qb[blocks]], qb[:blocks + 1]

    def fused_block_matrix(self, circ: Circuit, block: int) -> np.ndarray:
        arr, keep = ops_struct_array(circ)
        out = np.zeros(2 * 64 * 64, np.float64)
        dim = self.L.ref_fused_block_matrix(C.addressof(arr), len(circ.ops), block, out, out.size)
        del keep
        return out[:2 * dim * dim].view(np.complex128).reshape(dim, dim).copy()

    def run(self, circ: Circuit, fuse_gates=True, threads=0, statevector=True, shots=0, seed=0, targets=(),
            width=None, paulis=(), timing=False, engine="cpu"):
        """DenseEngine::execute (engine="cpu") or CudaDenseEngine::execute
        (engine="cuda", a RefLib on REF_CUDA_SO); returns dict(statevector,
        counts, terms, seconds)."""
        run_fn = self.L.ref_run_cuda if engine == "cuda" else self.L.ref_run_dense
        arr, keep = ops_struct_array(circ)
        n = circ.num_qubits
        sv = np.zeros(1 << n, np.complex128) if statevector else None
        t = np.asarray(targets, np.uint32).ravel()
        if width is None:
            width = int(max(t[1::2]) + 1) if len(t) else 0
        cap = max(shots, 1)
        outc = np.zeros(cap, np.uint64)
        cnt = np.zeros(cap, np.uint64)
        nout = np.array([cap], np.uint64)
        xs = np.array([p[0] for p in paulis] or [0], np.uint64)
        zs = np.array([p[1] for p in paulis] or [0], np.uint64)
        terms = np.zeros(2 * max(len(paulis), 1), np.float64)
        secs = np.zeros(1, np.float64)
        rc = run_fn(
            n, C.addressof(arr), len(circ.ops), circ.global_phase, 1 if fuse_gates else 0, threads,
            sv.ctypes.data if sv is not None else None, shots, seed, t.ctypes.data if len(t) else None,
            len(t) // 2, width, outc.ctypes.data if shots else None, cnt.ctypes.data, nout.ctypes.data,
            xs.ctypes.data, zs.ctypes.data, len(paulis), terms.ctypes.data if paulis else None, secs.ctypes.data)
        assert rc == 0, self.L.ref_last_error()
        del keep
        d = int(nout[0]) if shots else 0
        return {
            "statevector": sv,
            "counts": {int(o): int(c) for o, c in zip(outc[:d], cnt[:d])},
            "terms": terms[:2 * len(paulis)].view(np.complex128).copy() if paulis else None,
            "seconds": float(secs[0]),
        }

    def run_dm(self, circ: Circuit, threads=0, shots=0, seed=0, targets=(), width=None, paulis=()):
        """DensityMatrixEngine::execute; returns dict(counts, terms, seconds)."""
        arr, keep = ops_struct_array(circ)
        t = np.asarray(targets, np.uint32).ravel()
        if width is None:
            width = int(max(t[1::2]) + 1) if len(t) else 0
        cap = max(shots, 1)
        outc = np.zeros(cap, np.uint64)
        cnt = np.zeros(cap, np.uint64)
        nout = np.array([cap], np.uint64)
        xs = np.array([p[0] for p in paulis] or [0], np.uint64)
        zs = np.array([p[1] for p in paulis] or [0], np.uint64)
        terms = np.zeros(2 * max(len(paulis), 1), np.float64)
        secs = np.zeros(1, np.float64)
        rc = self.L.ref_run_dm(
            circ.num_qubits, C.addressof(arr), len(circ.ops), threads, shots, seed,
            t.ctypes.data if len(t) else None, len(t) // 2, width, outc.ctypes.data if shots else None,
            cnt.ctypes.data, nout.ctypes.data, xs.ctypes.data, zs.ctypes.data, len(paulis),
            terms.ctypes.data if paulis else None, secs.ctypes.data)
        assert rc == 0, self.L.ref_last_error()
        del keep
        d = int(nout[0]) if shots else 0
        return {
            "counts": {int(o): int(c) for o, c in zip(outc[:d], cnt[:d])},
            "terms": terms[:2 * len(paulis)].view(np.complex128).copy() if paulis else None,
            "seconds": float(secs[0]),
        }

    def pass_plan(self, circ: Circuit, chunk_qubits: int, window_qubits: int):
        """The chunked tier's pass plan over the circuit's fusion plan
        (build_pass_plan, or choose_pass_plan for chunk_qubits 0):
        (chunk_qubits, window_too_small, [(global_mask, first, end), ...])."""
        arr, keep = ops_struct_array(circ)
        out = np.zeros(1 << 20, np.uint64)
        k = self.L.ref_pass_plan(circ.num_qubits, C.addressof(arr), len(circ.ops), chunk_qubits, window_qubits,
                                 out.ctypes.data, out.size)
        assert k >= 0, self.L.ref_last_error()
        del keep
        w = [int(v) for v in out[:k]]
        return w[0], bool(w[1]), [tuple(w[3 + 3 * i:6 + 3 * i]) for i in range(w[2])]

    def run_trajectories(self, circ: Circuit, trajectories, seed, paulis=(), coefs=None, shots=0, targets=(),
                         width=None):
        """TrajectoryEngine::execute; returns dict(terms, standard_error, counts)."""
        arr, keep = ops_struct_array(circ)
        T = len(paulis)
        xs = np.array([p[0] for p in paulis] or [0], np.uint64)
        zs = np.array([p[1] for p in paulis] or [0], np.uint64)
        cs = np.ascontiguousarray(np.asarray(coefs if coefs is not None else [1.0] * max(T, 1), np.complex128))
        terms = np.zeros(2 * max(T, 1), np.float64)
        se = np.zeros(1, np.float64)
        t = np.asarray(targets, np.uint32).ravel()
        if width is None:
            width = int(max(t[1::2]) + 1) if len(t) else 0
        cap = max(shots, 1)
        outc = np.zeros(cap, np.uint64)
        cnt = np.zeros(cap, np.uint64)
        nout = np.array([cap], np.uint64)
        rc = self.L.ref_run_trajectories(circ.num_qubits, C.addressof(arr), len(circ.ops), trajectories, seed,
                                         xs.ctypes.data, zs.ctypes.data, cs.view(np.float64).ctypes.data, T,
                                         terms.ctypes.data, se.ctypes.data, shots,
                                         t.ctypes.data if len(t) else None, len(t) // 2, width,
                                         outc.ctypes.data, cnt.ctypes.data, nout.ctypes.data)
        assert rc == 0, self.L.ref_last_error()
        del keep
        d = int(nout[0]) if shots else 0
        return {"terms": terms[:2 * T].view(np.complex128).copy() if T else None,
                "standard_error": float(se[0]) if T else None,
                "counts": {int(o): int(c) for o, c in zip(outc[:d], cnt[:d])}}

    def run_plan(self, circ, plan, threads=0) -> np.ndarray:
        """The dense engine's fused sweep over an explicit plan (order,
        block_begin, block_qubits, qubits_begin): the statevector."""
        arr, keep = ops_struct_array(circ)
        order, bb, bq, qb = (np.ascontiguousarray(a, np.uint32) for a in plan)
        n = circ.num_qubits
        sv = np.zeros(1 << n, np.complex128)
        rc = self.L.ref_run_plan(n, C.addressof(arr), len(circ.ops), circ.global_phase, order.ctypes.data,
                                 bb.ctypes.data, bq.ctypes.data if bq.size else None, qb.ctypes.data, len(bb) - 1,
                                 threads, sv.ctypes.data)
        assert rc == 0, self.L.ref_last_error()
        del keep
        return sv

    def default_threads(self) -> int:
        return int(self.L.ref_default_threads())

    def kernel_isa(self) -> str:
        return "avx2" if self.L.ref_kernel_isa() else "baseline"
