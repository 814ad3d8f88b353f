"""ctypes binding of libmenos_b200.so (the C ABI in include/mb2.h).

The library is built in-tree (``python -m menos_b200.build``); importing this
module without it raises, so no caller can silently run without the CUDA
path.
"""
from __future__ import annotations

import ctypes as C
import os

from .circuit import MB2Op

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libmenos_b200.so")

MB2_OK = 0
ERRORS = {1: "invalid argument", 2: "resource exceeded", 3: "CUDA error", 4: "no sm_100 device",
          5: "timeout", 6: "unsupported", 7: "abandoned"}
C128, C64 = 0, 1
BATCH_MAX_TERMS = 64  # MB2_BATCH_MAX_TERMS


class SweepOptions(C.Structure):
    _fields_ = [("fuse_gates", C.c_int32), ("low_qubits", C.c_int32), ("tile_qubits", C.c_int32),
                ("per_gate", C.c_int32), ("c64_kernel", C.c_int32), ("fusion_width", C.c_int32)]


class SweepEstimate(C.Structure):
    _fields_ = [("blocks", C.c_uint64), ("passes", C.c_uint64), ("launches", C.c_uint64),
                ("device_bytes", C.c_uint64), ("h2d_bytes", C.c_uint64), ("work_units", C.c_uint64),
                ("fp64_ops_per_amp", C.c_uint64)]


BOUNDARY_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64)


class BatchOptions(C.Structure):
    _fields_ = [("precision", C.c_int32), ("fuse_gates", C.c_int32), ("tile_qubits", C.c_int32),
                ("reserved", C.c_int32)]


class BatchStats(C.Structure):
    _fields_ = [("passes", C.c_uint64), ("blocks", C.c_uint64), ("parametric_blocks", C.c_uint64),
                ("h2d_bytes", C.c_uint64), ("fp64_ops_per_amp", C.c_uint64)]


class ServerOptions(C.Structure):
    _fields_ = [("device_budget_bytes", C.c_uint64), ("slots", C.c_uint32), ("reserved", C.c_uint32)]


class Request(C.Structure):
    _fields_ = [("ops", C.POINTER(MB2Op)), ("num_ops", C.c_uint32), ("num_qubits", C.c_uint32),
                ("global_phase", C.c_double), ("fuse_gates", C.c_int32), ("output", C.c_int32),
                ("shots", C.c_uint64), ("seed", C.c_uint64), ("targets", C.c_void_p), ("num_targets", C.c_uint32),
                ("num_terms", C.c_uint32), ("x_masks", C.c_void_p), ("z_masks", C.c_void_p),
                ("coefs", C.c_void_p), ("precision", C.c_int32), ("reserved", C.c_uint32)]


class Completion(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("status", C.c_int32), ("reserved", C.c_uint32), ("value", C.c_double),
                ("num_outcomes", C.c_uint64), ("outcomes", C.POINTER(C.c_uint64)),
                ("counts", C.POINTER(C.c_uint64)), ("queue_seconds", C.c_double),
                ("latency_seconds", C.c_double)]


OUT_COUNTS, OUT_EXPECTATION = 1, 2


class Tuning(C.Structure):
    _fields_ = [("tile_qubits", C.c_uint32), ("tile_qubits_c64", C.c_uint32), ("pass_s_fixed", C.c_double),
                ("pass_s_per_amp", C.c_double), ("dense1_s_per_amp", C.c_double), ("diag_s_per_amp", C.c_double),
                ("pass_s_fixed_c64", C.c_double), ("pass_s_per_amp_c64", C.c_double), ("dense1_s_per_amp_c64", C.c_double),
                ("diag_s_per_amp_c64", C.c_double), ("probe_qubits", C.c_uint32), ("reserved", C.c_uint32)]


class SweepStats(C.Structure):
    _fields_ = [("blocks", C.c_uint64), ("passes", C.c_uint64), ("launches", C.c_uint64),
                ("fp64_ops_per_amp", C.c_uint64)]


# Exported symbol -> (restype, argtypes); the list the C-ABI tests check
# against include/mb2.h.
_VP = C.c_void_p
# mb2_ledger_charge_fn / mb2_ledger_release_fn
LEDGER_CHARGE = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_uint64)
LEDGER_RELEASE = C.CFUNCTYPE(None, C.c_void_p, C.c_uint64)

SIGNATURES = {
    "mb2_context_create": (C.c_int, [C.c_int, C.POINTER(_VP)]),
    "mb2_context_destroy": (C.c_int, [_VP]),
    "mb2_last_error": (C.c_int, [_VP, C.c_char_p, C.c_size_t]),
    "mb2_device_info": (C.c_int, [_VP, C.POINTER(C.c_int), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "mb2_sweep_batch": (C.c_int, [_VP, C.POINTER(MB2Op), C.c_uint32, C.c_uint32, _VP, C.c_uint32, C.c_uint32,
                                  _VP, _VP, _VP, C.c_uint32, C.POINTER(BatchOptions), _VP, _VP,
                                  C.POINTER(BatchStats)]),
    "mb2_server_create": (C.c_int, [_VP, C.POINTER(ServerOptions), C.POINTER(_VP)]),
    "mb2_server_submit": (C.c_int, [_VP, C.POINTER(Request), C.POINTER(C.c_uint64)]),
    "mb2_server_poll": (C.c_int, [_VP, C.POINTER(Completion), C.c_uint32, C.POINTER(C.c_uint32), C.c_uint32]),
    "mb2_server_release": (C.c_int, [_VP, C.c_uint64]),
    "mb2_server_stats": (C.c_int, [_VP, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                   C.POINTER(C.c_uint64)]),
    "mb2_server_destroy": (C.c_int, [_VP]),
    "mb2_server_set_ledger": (C.c_int, [_VP, _VP, _VP, _VP]),
    "mb2_probe_rates": (C.c_int, [_VP, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "mb2_kernel_launches": (C.c_int, [C.POINTER(C.c_uint64)]),
    "mb2_autotune": (C.c_int, [_VP, C.c_uint32, _VP]),
    "mb2_context_tuning": (C.c_int, [_VP, _VP]),
    "mb2_estimate_sweep_time": (C.c_int, [_VP, C.POINTER(MB2Op), C.c_uint32, C.POINTER(SweepOptions), C.c_uint32,
                                          C.c_int32, C.POINTER(C.c_double)]),
    "mb2_debug_pauli_groups": (C.c_int, [_VP, _VP, C.c_uint32, C.c_uint32, _VP, C.POINTER(C.c_uint64)]),
    "mb2_state_alloc": (C.c_int, [_VP, C.c_uint32, C.c_int, C.c_uint64, C.POINTER(_VP)]),
    "mb2_state_free": (C.c_int, [_VP]),
    "mb2_init": (C.c_int, [_VP, C.c_double]),
    "mb2_state_device_ptr": (C.c_int, [_VP, C.POINTER(_VP)]),
    "mb2_state_stream": (C.c_int, [_VP, C.POINTER(_VP)]),
    "mb2_apply_matrix": (C.c_int, [_VP, _VP, _VP, C.c_uint32]),
    "mb2_apply_matrix_generic": (C.c_int, [_VP, _VP, _VP, C.c_uint32]),
    "mb2_apply_program": (C.c_int, [_VP, C.POINTER(MB2Op), C.c_uint32, C.POINTER(SweepOptions)]),
    "mb2_apply_program_monitored": (C.c_int, [_VP, C.POINTER(MB2Op), C.c_uint32, C.POINTER(SweepOptions),
                                              BOUNDARY_FN, _VP]),
    "mb2_estimate_sweep": (C.c_int, [C.POINTER(MB2Op), C.c_uint32, C.POINTER(SweepOptions), C.c_uint32,
                                     C.POINTER(SweepEstimate)]),
    "mb2_last_sweep_stats": (C.c_int, [_VP, C.POINTER(SweepStats)]),
    "mb2_expectation": (C.c_int, [_VP, _VP, _VP, C.c_uint32, _VP]),
    "mb2_expectation_noalloc": (C.c_int, [_VP, C.c_uint32, _VP, _VP, C.c_uint32, _VP, _VP]),
    "mb2_norm": (C.c_int, [_VP, C.POINTER(C.c_double)]),
    "mb2_normalize": (C.c_int, [_VP, C.POINTER(C.c_double)]),
    "mb2_sample": (C.c_int, [_VP, C.c_uint64, C.c_uint64, _VP, C.c_uint32, _VP, _VP, C.POINTER(C.c_uint64)]),
    "mb2_norm_exact": (C.c_int, [_VP, C.POINTER(C.c_double)]),
    "mb2_state_alloc_host": (C.c_int, [_VP, C.c_uint32, C.c_uint64, C.POINTER(_VP)]),
    "mb2_state_host_ptr": (C.c_int, [_VP, C.POINTER(_VP)]),
    "mb2_trajectories": (C.c_int, [_VP, C.c_uint32, _VP, C.c_uint32, C.c_uint64, C.c_uint64, _VP, _VP, _VP,
                                   C.c_uint32, _VP, C.POINTER(C.c_double), C.c_uint64, _VP, C.c_uint32, _VP, _VP,
                                   C.POINTER(C.c_uint64)]),
    "mb2_dm_apply_program": (C.c_int, [_VP, C.c_uint32, _VP, C.c_uint32]),
    "mb2_dm_expectation": (C.c_int, [_VP, C.c_uint32, _VP, _VP, C.c_uint32, _VP]),
    "mb2_dm_sample": (C.c_int, [_VP, C.c_uint32, C.c_uint64, C.c_uint64, _VP, C.c_uint32, _VP, _VP,
                                C.POINTER(C.c_uint64)]),
    "mb2_dm_sample_readout": (C.c_int, [_VP, C.c_uint32, _VP, C.c_uint32, C.c_uint64, C.c_uint64, _VP, C.c_uint32,
                                        _VP, _VP, C.POINTER(C.c_uint64)]),
    "mb2_dm_sample_basis": (C.c_int, [_VP, C.c_uint32, _VP, C.c_uint64, _VP]),
    "mb2_apply_program_windowed": (C.c_int, [_VP, C.POINTER(MB2Op), C.c_uint32, C.POINTER(SweepOptions), C.c_uint32,
                                             C.c_uint32]),
    "mb2_window_plan": (C.c_int, [C.POINTER(MB2Op), C.c_uint32, C.POINTER(SweepOptions), C.c_uint32, C.c_uint32,
                                  C.c_uint32, _VP, C.POINTER(C.c_uint64)]),
    "mb2_trajectories_monitored": (C.c_int, [_VP, C.c_uint32, _VP, C.c_uint32, C.c_uint64, C.c_uint64, _VP, _VP,
                                             _VP, C.c_uint32, _VP, C.POINTER(C.c_double), C.c_uint64, _VP,
                                             C.c_uint32, _VP, _VP, C.POINTER(C.c_uint64), _VP, _VP]),
    "mb2_sample_basis": (C.c_int, [_VP, _VP, C.c_uint64, _VP]),
    "mb2_debug_tc_probe": (C.c_int, [_VP, _VP, _VP, _VP]),
    "mb2_fusion_plan": (C.c_int, [C.POINTER(MB2Op), C.c_uint32, C.POINTER(SweepOptions), _VP, _VP, _VP, _VP,
                                  C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "mb2_debug_run_plan": (C.c_int, [C.POINTER(MB2Op), C.c_uint32, C.POINTER(SweepOptions), C.c_uint32, C.c_int32,
                                     _VP, _VP]),
    "mb2_copy_out": (C.c_int, [_VP, _VP, C.c_uint64]),
    "mb2_copy_in": (C.c_int, [_VP, _VP, C.c_uint64]),
    "mb2_synchronize": (C.c_int, [_VP]),
    "mb2_gate_matrix": (C.c_int, [C.c_int32, _VP, _VP, C.c_uint32]),
    "mb2_debug_schedule": (C.c_int, [C.POINTER(MB2Op), C.c_uint32, C.POINTER(SweepOptions), C.c_uint32, _VP, _VP,
                                     _VP, _VP, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.c_int32]),
}

_lib = None


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libmenos_b200.so is not built ({LIB_PATH}); run python -m menos_b200.build")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class MB2Error(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


class ResourceExceeded(MB2Error):
    """The reference's common::ResourceExceeded (src/common/error.h:29-43)."""


def check(rc: int, ctx=None, what: str = "") -> None:
    if rc == MB2_OK:
        return
    msg = what
    if ctx is not None:
        buf = C.create_string_buffer(512)
        lib().mb2_last_error(ctx, buf, 512)
        msg = f"{what}: {buf.value.decode(errors='replace')}"
    if rc == 2:
        raise ResourceExceeded(rc, msg)
    raise MB2Error(rc, msg)
