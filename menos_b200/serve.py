"""Python face of the serving loop (mb2_server_*): submit circuit requests as
they arrive, poll completions.  The loop itself is C++
(menos_b200/csrc/serve.cpp)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import OUT_COUNTS, OUT_EXPECTATION, Completion, Request, ServerOptions, check, lib
from .circuit import Circuit, to_mb2_ops
from .engine import Context, Counts


class Server:
    def __init__(self, ctx: Context, budget_bytes: int = 0, slots: int = 0):
        self.ctx = ctx
        h = C.c_void_p()
        opts = ServerOptions(budget_bytes, slots, 0)
        check(lib().mb2_server_create(ctx.h, C.byref(opts), C.byref(h)), ctx.h, "mb2_server_create")
        self.h = h

    def submit(self, circ: Circuit, output: str = "expectation", shots: int = 0, seed: int = 0, targets=(),
               paulis=(), coefs=(), fuse_gates: bool = True, precision: int = _lib.C128) -> int:
        arr, keep = to_mb2_ops(circ)
        t = np.ascontiguousarray(np.asarray(targets, np.uint32).ravel())
        xs = np.ascontiguousarray([int(p[0]) for p in paulis] or [0], dtype=np.uint64)
        zs = np.ascontiguousarray([int(p[1]) for p in paulis] or [0], dtype=np.uint64)
        cs = np.ascontiguousarray(list(coefs) or [0.0], dtype=np.float64)
        req = Request()
        req.ops = arr
        req.num_ops = len(circ.ops)
        req.num_qubits = circ.num_qubits
        req.global_phase = circ.global_phase
        req.fuse_gates = 1 if fuse_gates else 0
        req.output = OUT_COUNTS if output == "counts" else OUT_EXPECTATION
        req.shots = shots
        req.seed = seed
        req.targets = t.ctypes.data if len(t) else None
        req.num_targets = len(t) // 2
        req.num_terms = len(paulis)
        req.x_masks = xs.ctypes.data
        req.z_masks = zs.ctypes.data
        req.coefs = cs.ctypes.data
        req.precision = precision
        ticket = C.c_uint64()
        check(lib().mb2_server_submit(self.h, C.byref(req), C.byref(ticket)), self.ctx.h, "mb2_server_submit")
        del keep
        return ticket.value

    def poll(self, timeout_ms: int = 100, capacity: int = 256):
        """Completed requests as dicts (ticket, status, value, counts, queue_s,
        latency_s); counts as a Counts mapping over numpy arrays (copied out
        of the completion before it is released, no per-outcome objects)."""
        buf = (Completion * capacity)()
        n = C.c_uint32()
        rc = lib().mb2_server_poll(self.h, buf, capacity, C.byref(n), timeout_ms)
        out = []
        for i in range(n.value):
            c = buf[i]
            counts = None
            if c.num_outcomes:
                k = int(c.num_outcomes)
                counts = Counts(np.ctypeslib.as_array(c.outcomes, shape=(k,)).copy(),
                                np.ctypeslib.as_array(c.counts, shape=(k,)).copy())
            out.append({"ticket": c.ticket, "status": c.status, "value": c.value, "counts": counts,
                        "queue_s": c.queue_seconds, "latency_s": c.latency_seconds})
            lib().mb2_server_release(self.h, c.ticket)
        if rc not in (_lib.MB2_OK, 5):
            check(rc, self.ctx.h, "mb2_server_poll")
        return out

    def set_ledger(self, charge, release) -> None:
        """Admission through a memory ledger: charge(bytes) -> bool is asked
        before a request is admitted (False keeps it pending), release(bytes)
        is called when its memory is freed.  Both run on server threads."""
        self._ledger = (_lib.LEDGER_CHARGE(lambda _u, b: 1 if charge(int(b)) else 0),
                        _lib.LEDGER_RELEASE(lambda _u, b: release(int(b))))
        check(lib().mb2_server_set_ledger(self.h, C.cast(self._ledger[0], C.c_void_p),
                                          C.cast(self._ledger[1], C.c_void_p), None),
              self.ctx.h, "mb2_server_set_ledger")

    def stats(self):
        p, f, hb, bb = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        lib().mb2_server_stats(self.h, C.byref(p), C.byref(f), C.byref(hb), C.byref(bb))
        return {"pending": p.value, "in_flight": f.value, "held_bytes": hb.value, "budget_bytes": bb.value}

    def close(self):
        if self.h:
            lib().mb2_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
