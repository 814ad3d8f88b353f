"""Python side of the engine: device contexts, device states and the
``B200DenseEngine`` that mirrors the reference's ``SimulationEngine``
interface for the dense statevector path
(include/menos/simulation_engine.h:322-367; request/result fields :141-234).

Everything computes through libmenos_b200.so; nothing here has a CPU path.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from collections.abc import Mapping
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import C128, C64, SweepOptions, SweepStats, check, lib
from .circuit import Circuit, to_mb2_ops


class Counts(Mapping):
    """Measurement counts as the engine returns them: outcome -> shots, in
    ascending outcome order, held as two numpy arrays (a million distinct
    outcomes cost no Python objects until they are read).  Compares equal
    to a dict with the same items."""

    def __init__(self, outcomes: np.ndarray, counts: np.ndarray):
        self.outcomes = outcomes
        self.counts = counts

    def __len__(self) -> int:
        return int(self.outcomes.size)

    def __iter__(self):
        return iter(self.outcomes.tolist())

    def __getitem__(self, key) -> int:
        i = int(np.searchsorted(self.outcomes, np.uint64(key)))
        if i < self.outcomes.size and int(self.outcomes[i]) == int(key):
            return int(self.counts[i])
        raise KeyError(key)

    def items(self):
        return zip(self.outcomes.tolist(), self.counts.tolist())

    def to_dict(self) -> dict:
        return dict(self.items())

    def __eq__(self, other):
        if isinstance(other, Counts):
            return np.array_equal(self.outcomes, other.outcomes) and np.array_equal(self.counts, other.counts)
        if isinstance(other, Mapping):
            return self.to_dict() == dict(other.items())
        return NotImplemented

    def __repr__(self) -> str:
        return f"Counts({len(self)} outcomes, {int(self.counts.sum())} shots)"


class Context:
    """One device (reference: DeviceInfo + DevicePool set-up,
    src/kernels/cuda/device_info.h:14-55)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        rc = lib().mb2_context_create(device, C.byref(h))
        if rc != _lib.MB2_OK:
            raise _lib.MB2Error(rc, f"mb2_context_create(device={device})")
        self.h = h
        self.device = device

    def tc_probe(self, rows: np.ndarray, matrix: np.ndarray) -> np.ndarray:
        """The tensor-core step alone (mb2_debug_tc_probe): rows (256 x 16
        complex64) times matrix^T (16 x 16 complex), split-FP16 on tcgen05."""
        r = np.ascontiguousarray(np.asarray(rows, np.complex64).reshape(256, 16))
        m = np.ascontiguousarray(np.asarray(matrix, np.complex128).reshape(16, 16))
        out = np.zeros((256, 16), np.complex64)
        check(lib().mb2_debug_tc_probe(self.h, r.ctypes.data, m.ctypes.data, out.ctypes.data), self.h,
              "mb2_debug_tc_probe")
        return out

    def close(self) -> None:
        if self.h:
            lib().mb2_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def probe_rates(self):
        """(FP64 instructions/s, device copy GB/s) measured on this device."""
        f, c = C.c_double(), C.c_double()
        check(lib().mb2_probe_rates(self.h, C.byref(f), C.byref(c)), self.h, "probe_rates")
        return f.value, c.value

    def autotune(self, probe_qubits: int = 0) -> dict:
        """Measures the best tile widths and the time model's costs on this
        device (mb2_autotune); they become this context's defaults."""
        t = _lib.Tuning()
        check(lib().mb2_autotune(self.h, probe_qubits, C.byref(t)), self.h, "mb2_autotune")
        return {f: getattr(t, f) for f, _ in t._fields_ if f != "reserved"}

    def tuning(self) -> dict:
        t = _lib.Tuning()
        check(lib().mb2_context_tuning(self.h, C.byref(t)), self.h, "mb2_context_tuning")
        return {f: getattr(t, f) for f, _ in t._fields_ if f != "reserved"}

    def estimate_time(self, circ: Circuit, precision: int = C128, fuse_gates: bool = True,
                      tile_qubits: int = 0) -> float:
        """Seconds the sweep of circ would take here, from the tuned time model."""
        arr, keep = to_mb2_ops(circ)
        opts = SweepOptions(1 if fuse_gates else 0, 0, tile_qubits, 0)
        sec = C.c_double()
        check(lib().mb2_estimate_sweep_time(self.h, arr, len(circ.ops), C.byref(opts), circ.num_qubits, precision,
                                            C.byref(sec)), self.h, "mb2_estimate_sweep_time")
        del keep
        return sec.value

    def info(self):
        sm, tot, fr = C.c_int(), C.c_uint64(), C.c_uint64()
        check(lib().mb2_device_info(self.h, C.byref(sm), C.byref(tot), C.byref(fr)), self.h, "device_info")
        return {"sm_count": sm.value, "total_bytes": tot.value, "free_bytes": fr.value}


class DeviceState:
    """A statevector in device memory (reference: DeviceBuffer,
    src/kernels/cuda/device_buffer.h:25-55)."""

    def __init__(self, ctx: Context, num_qubits: int, precision: int = C128, budget_bytes: int = 2 ** 64 - 1,
                 host: bool = False):
        """host=True: a complex128 state in pinned, mapped host memory
        (mb2_state_alloc_host), for states above the device's memory."""
        h = C.c_void_p()
        if host:
            if precision != C128:
                raise ValueError("host-resident states are complex128")
            check(lib().mb2_state_alloc_host(ctx.h, num_qubits, min(budget_bytes, 2 ** 64 - 1), C.byref(h)),
                  ctx.h, "mb2_state_alloc_host")
        else:
            check(lib().mb2_state_alloc(ctx.h, num_qubits, precision, min(budget_bytes, 2 ** 64 - 1), C.byref(h)),
                  ctx.h, "mb2_state_alloc")
        self.ctx = ctx
        self.h = h
        self.n = num_qubits
        self.precision = precision

    def free(self) -> None:
        if self.h:
            lib().mb2_state_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def stream_handle(self) -> int:
        """The cudaStream_t this state's work is queued on (as an int)."""
        h = C.c_void_p()
        self._chk(lib().mb2_state_stream(self.h, C.byref(h)), "mb2_state_stream")
        return h.value or 0

    def _chk(self, rc, what):
        check(rc, self.ctx.h, what)

    def init(self, global_phase: float = 0.0) -> None:
        self._chk(lib().mb2_init(self.h, global_phase), "mb2_init")

    def apply_matrix(self, matrix, operands, generic: bool = False) -> None:
        m = np.ascontiguousarray(np.asarray(matrix, np.complex128)).view(np.float64).ravel()
        q = np.ascontiguousarray(np.asarray(operands, np.uint32))
        f = lib().mb2_apply_matrix_generic if generic else lib().mb2_apply_matrix
        self._chk(f(self.h, m.ctypes.data, q.ctypes.data, len(q)), "mb2_apply_matrix")

    def apply_program(self, circ: Circuit, fuse_gates: bool = True, tile_qubits: int = 0,
                      per_gate: bool = False, low_qubits: int = 0, c64_kernel: str = "auto",
                      fusion_width: int = 0) -> SweepStats:
        """c64_kernel (complex64 states): "tensor" -- each phase's gates as one
        split-FP16 tensor-core GEMM wherever a pass allows; "simt" -- FP32
        gates one by one; "auto" -- tensor cores for states of more than 2^24
        amplitudes, SIMT below.  fusion_width (with fuse_gates): 0 -- the
        reference's containment rule; 2..6 -- blocks of up to that many qubits
        (fusion_plan gives the plan)."""
        arr, keep = to_mb2_ops(circ)
        kernels = {"auto": 0, "simt": 1, "tensor": 2}
        if c64_kernel not in kernels:
            raise ValueError("c64_kernel is 'auto', 'tensor' or 'simt'")
        opts = SweepOptions(1 if fuse_gates else 0, low_qubits, tile_qubits, 1 if per_gate else 0,
                            kernels[c64_kernel], fusion_width)
        self._chk(lib().mb2_apply_program(self.h, arr, len(circ.ops), C.byref(opts)), "mb2_apply_program")
        del keep
        return self.stats()

    def apply_program_windowed(self, circ: Circuit, window_qubits: int, chunk_qubits: int = 0,
                               fuse_gates: bool = True) -> SweepStats:
        """A host-resident state swept through device windows of
        2^window_qubits amplitudes (mb2_apply_program_windowed: the
        reference's chunked tier on the copy engines; chunk_qubits 0 chooses
        the chunk as the reference does).  stats.passes counts window
        passes."""
        arr, keep = to_mb2_ops(circ)
        opts = SweepOptions(1 if fuse_gates else 0, 0, 0, 0, 0, 0)
        self._chk(lib().mb2_apply_program_windowed(self.h, arr, len(circ.ops), C.byref(opts), window_qubits,
                                                   chunk_qubits), "mb2_apply_program_windowed")
        del keep
        return self.stats()

    def stats(self) -> SweepStats:
        s = SweepStats()
        self._chk(lib().mb2_last_sweep_stats(self.h, C.byref(s)), "stats")
        return s

    def expectation(self, paulis: Sequence[tuple]) -> np.ndarray:
        """paulis: (x_mask, z_mask) pairs -> complex128 array (coefficients not applied)."""
        if len(paulis) == 0:
            return np.zeros(0, np.complex128)
        xs = np.ascontiguousarray([int(p[0]) for p in paulis], dtype=np.uint64)
        zs = np.ascontiguousarray([int(p[1]) for p in paulis], dtype=np.uint64)
        out = np.zeros(2 * len(paulis), np.float64)
        self._chk(lib().mb2_expectation(self.h, xs.ctypes.data, zs.ctypes.data, len(paulis), out.ctypes.data),
                  "mb2_expectation")
        return out.view(np.complex128).copy()

    def normalize(self) -> float:
        """complex64: rescale to unit norm (returns the norm before)."""
        v = C.c_double()
        self._chk(lib().mb2_normalize(self.h, C.byref(v)), "mb2_normalize")
        return v.value

    def norm_exact(self) -> float:
        """The reference's sequential sum of |a|^2, bit for bit."""
        v = C.c_double()
        self._chk(lib().mb2_norm_exact(self.h, C.byref(v)), "mb2_norm_exact")
        return v.value

    def norm(self) -> float:
        v = C.c_double()
        self._chk(lib().mb2_norm(self.h, C.byref(v)), "mb2_norm")
        return v.value

    def sample(self, shots: int, seed: int, targets) -> "Counts":
        t = np.ascontiguousarray(np.asarray(targets, np.uint32).ravel())
        cap = max(int(shots), 1)
        outc = np.zeros(cap, np.uint64)
        cnt = np.zeros(cap, np.uint64)
        nout = C.c_uint64(cap)
        self._chk(lib().mb2_sample(self.h, shots, seed, t.ctypes.data if len(t) else None, len(t) // 2,
                                   outc.ctypes.data, cnt.ctypes.data, C.byref(nout)), "mb2_sample")
        d = nout.value
        return Counts(outc[:d].copy(), cnt[:d].copy())

    def copy_out(self) -> np.ndarray:
        dt = np.complex128 if self.precision == C128 else np.complex64
        out = np.zeros(1 << self.n, dt)
        self._chk(lib().mb2_copy_out(self.h, out.ctypes.data, out.size), "mb2_copy_out")
        return out

    def copy_in(self, amps: np.ndarray) -> None:
        dt = np.complex128 if self.precision == C128 else np.complex64
        a = np.ascontiguousarray(amps, dtype=dt)
        self._chk(lib().mb2_copy_in(self.h, a.ctypes.data, a.size), "mb2_copy_in")

    def synchronize(self) -> None:
        self._chk(lib().mb2_synchronize(self.h), "mb2_synchronize")


def trajectories(ctx: Context, circ: Circuit, count: int, seed: int, paulis=(), coefs=None, shots: int = 0,
                 targets=()) -> dict:
    """mb2_trajectories: the reference's trajectory engine on the device.
    Returns {"terms": complex means per Pauli term, "standard_error": of
    sum coef_t <P_t> (coefs default 1), "counts": Counts or None}."""
    arr, keep = to_mb2_ops(circ)
    T = len(paulis)
    xs = np.ascontiguousarray([int(p[0]) for p in paulis] or [0], dtype=np.uint64)
    zs = np.ascontiguousarray([int(p[1]) for p in paulis] or [0], dtype=np.uint64)
    cs = np.ascontiguousarray(np.asarray(coefs if coefs is not None else [1.0] * max(T, 1), np.complex128))
    means = np.zeros(2 * max(T, 1), np.float64)
    se = C.c_double(0.0)
    t = np.ascontiguousarray(np.asarray(targets, np.uint32).ravel())
    cap = max(int(shots), 1)
    outc = np.zeros(cap, np.uint64)
    cnt = np.zeros(cap, np.uint64)
    nout = C.c_uint64(cap)
    check(lib().mb2_trajectories(ctx.h, circ.num_qubits, arr, len(circ.ops), count, seed, xs.ctypes.data,
                                 zs.ctypes.data, cs.view(np.float64).ctypes.data, T, means.ctypes.data,
                                 C.byref(se), shots, t.ctypes.data if len(t) else None, len(t) // 2,
                                 outc.ctypes.data, cnt.ctypes.data, C.byref(nout)), ctx.h, "mb2_trajectories")
    del keep
    d = nout.value if shots else 0
    return {"terms": means[:2 * T].view(np.complex128).copy() if T else None,
            "standard_error": se.value if T else None,
            "counts": Counts(outc[:d].copy(), cnt[:d].copy()) if shots else None}


class DensityMatrix:
    """A density matrix of n qubits on the device: the reference's
    density-matrix engine (src/engines/density_matrix/
    density_matrix_engine.cpp).  rho is a complex128 state of 2n qubits,
    entry (r, c) at r | c << n; gates act as U on the row qubits and conj(U)
    on the column qubits, channels as their superoperators."""

    def __init__(self, ctx: Context, num_qubits: int, budget_bytes: int = 2 ** 64 - 1):
        if not 1 <= num_qubits <= 15:
            raise ValueError("a density matrix holds 1..15 qubits")
        self.n = num_qubits
        self.state = DeviceState(ctx, 2 * num_qubits, C128, budget_bytes)

    def _chk(self, rc, what):
        check(rc, self.state.ctx.h, what)

    def init(self) -> None:
        """|0..0><0..0| (a global phase cancels in rho)."""
        self.state.init(0.0)

    def apply(self, circ: Circuit) -> None:
        if circ.num_qubits != self.n:
            raise ValueError("circuit and density matrix differ in qubit count")
        arr, keep = to_mb2_ops(circ)
        self._chk(lib().mb2_dm_apply_program(self.state.h, self.n, arr, len(circ.ops)), "mb2_dm_apply_program")
        del keep

    def expectation(self, paulis: Sequence[tuple]) -> np.ndarray:
        """Tr(P rho) per (x_mask, z_mask) pair -> complex128 array."""
        if len(paulis) == 0:
            return np.zeros(0, np.complex128)
        xs = np.ascontiguousarray([int(p[0]) for p in paulis], dtype=np.uint64)
        zs = np.ascontiguousarray([int(p[1]) for p in paulis], dtype=np.uint64)
        out = np.zeros(2 * len(paulis), np.float64)
        self._chk(lib().mb2_dm_expectation(self.state.h, self.n, xs.ctypes.data, zs.ctypes.data, len(paulis),
                                           out.ctypes.data), "mb2_dm_expectation")
        return out.view(np.complex128).copy()

    def sample(self, shots: int, seed: int, targets, circuit: Circuit | None = None) -> "Counts":
        """Counts of rho's diagonal (the reference's samplers).  circuit:
        the measurements whose readout errors record the bits (the last
        measurement of each target's clbit, mb2_dm_sample_readout)."""
        t = np.ascontiguousarray(np.asarray(targets, np.uint32).ravel())
        cap = max(int(shots), 1)
        outc = np.zeros(cap, np.uint64)
        cnt = np.zeros(cap, np.uint64)
        nout = C.c_uint64(cap)
        if circuit is not None:
            arr, keep = to_mb2_ops(circuit)
            self._chk(lib().mb2_dm_sample_readout(self.state.h, self.n, arr, len(circuit.ops), shots, seed,
                                                  t.ctypes.data if len(t) else None, len(t) // 2,
                                                  outc.ctypes.data, cnt.ctypes.data, C.byref(nout)),
                      "mb2_dm_sample_readout")
            del keep
        else:
            self._chk(lib().mb2_dm_sample(self.state.h, self.n, shots, seed, t.ctypes.data if len(t) else None,
                                          len(t) // 2, outc.ctypes.data, cnt.ctypes.data, C.byref(nout)),
                      "mb2_dm_sample")
        d = nout.value
        return Counts(outc[:d].copy(), cnt[:d].copy())

    def matrix(self) -> np.ndarray:
        """rho as a (2^n, 2^n) array, rho[r, c]."""
        dim = 1 << self.n
        return self.state.copy_out().reshape(dim, dim).T.copy()

    def free(self) -> None:
        self.state.free()


def sweep_batch(ctx: Context, circ: Circuit, params, paulis, coefs, fuse_gates: bool = False, tile_qubits: int = 0,
                want_states: bool = False, precision: int = C128):
    """mb2_sweep_batch: <H> per binding for params[b] (one row per binding,
    the circuit's parameter slots in op order).  Returns (values, states or
    None, stats).  precision C64: complex64 states (FP32 gates, FP64
    reductions); states are returned promoted to complex128."""
    params = np.ascontiguousarray(np.asarray(params, np.float64))
    if params.ndim == 1:
        params = params.reshape(1, -1)
    B, ppb = params.shape
    arr, keep = to_mb2_ops(circ)
    xs = np.ascontiguousarray([int(p[0]) for p in paulis] or [0], dtype=np.uint64)
    zs = np.ascontiguousarray([int(p[1]) for p in paulis] or [0], dtype=np.uint64)
    cs = np.ascontiguousarray(list(coefs) or [0.0], dtype=np.float64)
    out = np.zeros(B, np.float64)
    states = np.zeros((B, 1 << circ.num_qubits), np.complex128) if want_states else None
    opts = _lib.BatchOptions(precision, 1 if fuse_gates else 0, tile_qubits, 0)
    stats = _lib.BatchStats()
    check(lib().mb2_sweep_batch(ctx.h, arr, len(circ.ops), circ.num_qubits, params.ctypes.data, ppb, B,
                                xs.ctypes.data, zs.ctypes.data, cs.ctypes.data, len(paulis), C.byref(opts),
                                out.ctypes.data, states.ctypes.data if want_states else None, C.byref(stats)),
          ctx.h, "mb2_sweep_batch")
    del keep
    return out, states, stats


# ---------------------------------------------------------------------------
# The SimulationEngine mirror.
# ---------------------------------------------------------------------------
@dataclasses.dataclass
class PauliTerm:
    x_mask: int
    z_mask: int
    coefficient: complex = 1.0


@dataclasses.dataclass
class EngineExecutionRequest:
    """menos::EngineExecutionRequest (include/menos/simulation_engine.h:141-198),
    the fields a dense engine reads."""
    num_qubits: int
    operations: Circuit
    want_statevector: bool = False
    want_counts: bool = False
    want_expectation: bool = False
    shots: int = 0
    measure_targets: Sequence[tuple] = ()
    bitstring_width: int = 0
    seed: int = 0
    global_phase: float = 0.0
    budget_bytes: int = 2 ** 64 - 1
    is_sole_region: bool = True
    observable: Optional[Sequence[PauliTerm]] = None
    fuse_gates: bool = True


@dataclasses.dataclass
class EngineExecutionResult:
    """menos::EngineExecutionResult (simulation_engine.h:227-236)."""
    statevector: Optional[np.ndarray] = None
    counts: Optional[dict] = None
    expectation_terms: Optional[np.ndarray] = None
    actual_bytes: int = 0
    sweep: Optional[dict] = None


class B200DenseEngine:
    """The dense statevector engine on one B200: {Dense, Cuda, InMemory}
    (the triple src/plan/execution_engines.cpp:37-45 resolves)."""

    def __init__(self, device: int = 0, tile_qubits: int = 0, fusion_width: int = 0):
        self.ctx = Context(device)
        self.tile_qubits = tile_qubits
        self.fusion_width = fusion_width

    def name(self) -> str:
        return "dense_b200"

    def engine_id(self) -> str:
        return "dense"

    def backend(self) -> str:
        return "cuda"

    def tier(self) -> str:
        return "in_memory"

    def capabilities(self) -> dict:
        return {"counts": True, "statevector": True, "expectation": True}

    def execute(self, req: EngineExecutionRequest) -> EngineExecutionResult:
        """CudaDenseEngine::execute's contract
        (src/engines/dense_cuda/cuda_dense_engine.cpp:325-412)."""
        for oc, *_ in req.operations.ops:
            if oc > 22 or oc < 0:
                raise _lib.MB2Error(6, "unsupported operation")
        st = DeviceState(self.ctx, req.num_qubits, C128, req.budget_bytes)
        try:
            st.init(req.global_phase)
            stats = st.apply_program(req.operations, fuse_gates=req.fuse_gates, tile_qubits=self.tile_qubits,
                                     fusion_width=self.fusion_width)
            res = EngineExecutionResult(actual_bytes=16 << req.num_qubits,
                                        sweep={"blocks": stats.blocks, "passes": stats.passes,
                                               "launches": stats.launches})
            if req.want_expectation:
                terms = list(req.observable or [])
                res.expectation_terms = st.expectation([(t.x_mask, t.z_mask) for t in terms])
            if req.want_counts:
                res.counts = st.sample(req.shots, req.seed, list(req.measure_targets))
            if req.want_statevector:
                res.statevector = st.copy_out()
            return res
        finally:
            st.free()


def fusion_plan(circ: Circuit, fusion_width: int = 0):
    """The fusion plan a sweep applies (mb2_fusion_plan), as the reference's
    ir::FusionPlan arrays: (order, block_begin, block_qubits, qubits_begin)."""
    arr, keep = to_mb2_ops(circ)
    n = len(circ.ops)
    order = np.zeros(max(n, 1), np.uint32)
    bb = np.zeros(n + 2, np.uint32)
    qb = np.zeros(n + 2, np.uint32)
    bq = np.zeros(max(6 * n, 1), np.uint32)
    nb = C.c_uint64(n + 1)
    nq = C.c_uint64(bq.size)
    opts = SweepOptions(1, 0, 0, 0, 0, fusion_width)
    rc = lib().mb2_fusion_plan(arr, n, C.byref(opts), order.ctypes.data, bb.ctypes.data, bq.ctypes.data,
                               qb.ctypes.data, C.byref(nb), C.byref(nq))
    check(rc, None, "mb2_fusion_plan")
    del keep
    b = nb.value
    return order[:n].copy(), bb[:b + 1].copy(), bq[:nq.value].copy(), qb[:b + 1].copy()
