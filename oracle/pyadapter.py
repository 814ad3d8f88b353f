"""TEST INFRASTRUCTURE: ctypes binding of _ref/libmenos_adapter.so.

The library (oracle/Makefile) holds the reference-side binding of this
engine -- menos_b200/integration/b200_dense_engine.cpp, the
menos::SimulationEngine MENOS would register -- beside the reference's own
CPU DenseEngine, both driven through adapter_harness.cpp.  Tests use it to
run the reference's CPU/CUDA differential cases against the adapter itself.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from pyoracle import ops_struct_array

HERE = os.path.dirname(os.path.abspath(__file__))
ADAPTER_SO = os.path.join(HERE, "_ref", "libmenos_adapter.so")

REFERENCE_CPU = 0   # engines::dense::DenseEngine
B200 = 1            # engines::dense_b200::B200DenseEngine (the adapter)
REFERENCE_DM = 2    # engines::density_matrix::DensityMatrixEngine
B200_DM = 3         # engines::dense_b200::b200_density_matrix_engine()
REFERENCE_TRAJ = 4  # engines::trajectory::TrajectoryEngine
B200_TRAJ = 5       # engines::dense_b200::b200_trajectory_engine()

OK, RESOURCE_EXCEEDED, INTERNAL_ERROR, OTHER = 0, 1, 2, 3


class _Request(C.Structure):
    _fields_ = [("num_qubits", C.c_uint32), ("num_ops", C.c_uint32), ("ops", C.c_void_p),
                ("fuse_gates", C.c_int32), ("want_statevector", C.c_int32), ("want_counts", C.c_int32),
                ("want_expectation", C.c_int32), ("is_sole_region", C.c_int32), ("reserved", C.c_int32),
                ("shots", C.c_uint64), ("seed", C.c_uint64), ("targets", C.c_void_p),
                ("num_targets", C.c_uint32), ("bitstring_width", C.c_uint32), ("global_phase", C.c_double),
                ("budget_bytes", C.c_uint64), ("x_masks", C.c_void_p), ("z_masks", C.c_void_p),
                ("num_terms", C.c_uint32), ("reserved2", C.c_uint32), ("abandon_at", C.c_int64),
                ("trajectories", C.c_uint64), ("coefs", C.c_void_p)]


class _Result(C.Structure):
    _fields_ = [("statevector", C.c_void_p), ("outcomes", C.c_void_p), ("counts", C.c_void_p),
                ("capacity", C.c_uint64), ("num_outcomes", C.c_uint64), ("expectation", C.c_void_p),
                ("draws", C.c_uint64), ("draw_seed", C.c_uint64), ("drawn", C.c_void_p),
                ("actual_bytes", C.c_uint64), ("peak_host", C.c_uint64), ("peak_device", C.c_uint64),
                ("monitor_calls", C.c_uint64), ("has_statevector", C.c_int32), ("has_counts", C.c_int32),
                ("has_sampler", C.c_int32), ("has_expectation", C.c_int32), ("seconds", C.c_double),
                ("standard_error", C.c_double), ("statistical", C.c_int32), ("reserved", C.c_int32)]


class AdapterHarness:
    def __init__(self, path: str = ADAPTER_SO):
        self.L = C.CDLL(path)
        self.L.ah_execute.restype = C.c_int
        self.L.ah_execute.argtypes = [C.c_int, C.POINTER(_Request), C.POINTER(_Result), C.c_char_p, C.c_size_t]
        self.L.ah_estimate.restype = C.c_int
        self.L.ah_estimate.argtypes = [C.c_int, C.POINTER(_Request), C.c_void_p, C.c_char_p, C.c_size_t]
        self.L.ah_calibration.restype = C.c_int
        self.L.ah_calibration.argtypes = [C.c_void_p]
        self.L.ah_serve_with_ledger.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_void_p]
        self.L.ah_serve_with_ledger.restype = C.c_int

    def _request(self, circ, keep, *, fuse=True, statevector=False, shots=0, seed=0, targets=(), width=None,
                 sole=True, paulis=(), global_phase=None, budget=1 << 40, abandon_at=-1, trajectories=0,
                 coefs=None):
        arr, mats = ops_struct_array(circ)
        keep += [arr, mats]
        t = np.ascontiguousarray(np.asarray(targets, np.uint32).ravel())
        keep.append(t)
        if width is None:
            width = int(max(t[1::2]) + 1) if len(t) else 0
        xs = np.ascontiguousarray(np.array([p[0] for p in paulis] or [0], np.uint64))
        zs = np.ascontiguousarray(np.array([p[1] for p in paulis] or [0], np.uint64))
        keep += [xs, zs]
        rq = _Request()
        rq.num_qubits = circ.num_qubits
        rq.num_ops = len(circ.ops)
        rq.ops = C.addressof(arr)
        rq.fuse_gates = 1 if fuse else 0
        rq.want_statevector = 1 if statevector else 0
        rq.want_counts = 1 if shots else 0
        rq.want_expectation = 1 if paulis else 0
        rq.is_sole_region = 1 if sole else 0
        rq.shots = shots
        rq.seed = seed
        rq.targets = t.ctypes.data if len(t) else None
        rq.num_targets = len(t) // 2
        rq.bitstring_width = width
        rq.global_phase = circ.global_phase if global_phase is None else global_phase
        rq.budget_bytes = budget
        rq.x_masks = xs.ctypes.data
        rq.z_masks = zs.ctypes.data
        rq.num_terms = len(paulis)
        rq.abandon_at = abandon_at
        rq.trajectories = trajectories
        if coefs is not None:
            cs = np.ascontiguousarray(np.asarray(coefs, np.complex128))
            keep.append(cs)
            rq.coefs = cs.ctypes.data
        return rq

    def execute(self, engine: int, circ, *, draws: int = 0, draw_seed: int = 0, **kw) -> dict:
        """EngineExecutionRequest through `engine`; returns rc, error and every output."""
        keep: list = []
        rq = self._request(circ, keep, **kw)
        n = circ.num_qubits
        sv = np.zeros(1 << n, np.complex128) if rq.want_statevector else None
        cap = max(int(rq.shots), draws, 1)
        outc = np.zeros(cap, np.uint64)
        cnt = np.zeros(cap, np.uint64)
        drawn = np.zeros(cap, np.uint64)
        terms = np.zeros(max(int(rq.num_terms), 1), np.complex128)
        res = _Result()
        res.statevector = sv.ctypes.data if sv is not None else None
        res.outcomes = outc.ctypes.data
        res.counts = cnt.ctypes.data
        res.capacity = cap
        res.expectation = terms.ctypes.data
        res.draws = draws
        res.draw_seed = draw_seed
        res.drawn = drawn.ctypes.data if draws else None
        err = C.create_string_buffer(1024)
        rc = self.L.ah_execute(engine, C.byref(rq), C.byref(res), err, len(err))
        d = int(res.num_outcomes)
        return {
            "rc": rc,
            "error": err.value.decode(errors="replace"),
            "statevector": sv if res.has_statevector else None,
            "counts": {int(o): int(c) for o, c in zip(outc[:d], cnt[:d])} if res.has_counts else None,
            "terms": terms[:int(rq.num_terms)].copy() if res.has_expectation else None,
            "has_sampler": bool(res.has_sampler),
            "drawn": drawn[:draws].copy() if (draws and res.has_sampler) else None,
            "actual_bytes": int(res.actual_bytes),
            "peak_host": int(res.peak_host),
            "peak_device": int(res.peak_device),
            "monitor_calls": int(res.monitor_calls),
            "seconds": float(res.seconds),
            "standard_error": float(res.standard_error) if res.standard_error >= 0 else None,
            "statistical": bool(res.statistical),
        }

    def estimate(self, engine: int, circ, **kw) -> dict:
        keep: list = []
        rq = self._request(circ, keep, **kw)
        out = np.zeros(8, np.uint64)
        reason = C.create_string_buffer(1024)
        rc = self.L.ah_estimate(engine, C.byref(rq), out.ctypes.data, reason, len(reason))
        assert rc == 0, reason.value
        keys = ["feasible", "peak_bytes", "work_units", "device_bytes", "h2d_bytes", "d2h_bytes", "launches",
                "host_passes"]
        d = {k: int(v) for k, v in zip(keys, out)}
        d["feasible"] = bool(d["feasible"])
        d["reason"] = reason.value.decode(errors="replace")
        return d

    def serve_with_ledger(self, qubits, slots, device_limit) -> dict:
        """The serving loop admitting through the adapter's ServerLedger."""
        q = np.ascontiguousarray(qubits, np.uint32)
        out = np.zeros(4, np.uint64)
        rc = self.L.ah_serve_with_ledger(q.ctypes.data, len(q), slots, device_limit, out.ctypes.data)
        assert rc == 0, rc
        return dict(zip(["peak_device_bytes", "live_device_bytes", "ok", "completed"], (int(v) for v in out)))

    def calibration(self) -> dict:
        out = np.zeros(8, np.float64)
        self.L.ah_calibration(out.ctypes.data)
        keys = ["present", "device_total_bytes", "device_available_bytes", "h2d_bytes_per_s", "d2h_bytes_per_s",
                "kernel_launch_seconds", "execution_seconds", "device_work_units_per_second"]
        return dict(zip(keys, out.tolist()))
