"""Qiskit-shaped Estimator and Sampler primitives over the B200 engine, batched.

The reference's primitives (python/menos/qiskit/estimator.py:86-156,
sampler.py:96-133) run one ``menos.run`` per observable of a pub and one per
pub, and refuse parameterised circuits.  These take the same pub shapes --
duck-typed, since they need no qiskit: a circuit (this package's
``Circuit``), observables, optional parameter values, precision / shots --
and batch them:

* Estimator: every observable of a pub comes from ONE device state (one
  sweep, one grouped expectation pass over the union of the observables'
  Pauli terms); a pub with parameter values runs all its bindings in one
  batched sweep (``mb2_sweep_batch``) per observable; pubs run concurrently,
  each on its own state and stream.
* Sampler: every pub (every binding of a parameterised pub) is a request of
  the serving loop (``mb2_server_*``), so the requests overlap on the device.

Observables are read as the reference's ``convert_observable`` reads a
``SparsePauliOp`` (``_observable_convert.py:15-51``): per term the x/z bit
arrays (bit j = qubit j, the phase of Y folded into the coefficient, i.e.
the convention P = i^{|x&z|} X^x Z^z) and a complex coefficient; a Pauli
label string is read Qiskit's way (the last character is qubit 0).  The
estimate is the real part of sum_t coef_t <P_t>, as the reference's
(estimator.py:145-148).  Parameter values for a pub: an array of shape
(*B, P) whose last axis gives every parameterised gate's parameters in op
order (the slots ``mb2_sweep_batch`` takes); the result shape is the
broadcast of B with the observables' shape.
"""
from __future__ import annotations

import concurrent.futures
import secrets
from typing import Any, Sequence

import numpy as np

from . import _lib
from .circuit import NUM_PARAMS, OP, Circuit
from .engine import Context, DeviceState, sweep_batch

_PAULI_BITS = {"I": (0, 0), "X": (1, 0), "Z": (0, 1), "Y": (1, 1)}
# The batched sweep's state sizes (include/mb2.h, mb2_sweep_batch).
_BATCH_MIN_QUBITS, _BATCH_MAX_QUBITS = 4, 16


def label_masks(label: str) -> tuple[int, int]:
    """A Pauli label (Qiskit order: label[-1] is qubit 0) as (x, z) masks."""
    x = z = 0
    for q, ch in enumerate(reversed(label.upper())):
        if ch not in _PAULI_BITS:
            raise ValueError(f"not a Pauli label: {label!r}")
        bx, bz = _PAULI_BITS[ch]
        x |= bx << q
        z |= bz << q
    return x, z


def observable_terms(obs: Any, num_qubits: int) -> list[tuple[int, int, complex]]:
    """One observable as (x_mask, z_mask, coefficient) terms.  Accepts a
    SparsePauliOp-like object (``.paulis.x`` / ``.paulis.z`` boolean arrays,
    ``.coeffs``), a dict {label: coeff}, a sequence of (label, coeff) or of
    (x, z, coeff), or a single label."""
    if hasattr(obs, "paulis") and hasattr(obs, "coeffs"):
        xb, zb = np.asarray(obs.paulis.x, bool), np.asarray(obs.paulis.z, bool)
        out = []
        for i in range(len(obs.coeffs)):
            x = sum(1 << q for q in range(num_qubits) if xb[i][q])
            z = sum(1 << q for q in range(num_qubits) if zb[i][q])
            out.append((x, z, complex(obs.coeffs[i])))
        return out
    if isinstance(obs, str):
        return [(*label_masks(obs), 1.0 + 0j)]
    items = obs.items() if isinstance(obs, dict) else obs
    out = []
    for item in items:
        if len(item) == 3:
            out.append((int(item[0]), int(item[1]), complex(item[2])))
        else:
            label, coeff = item
            out.append((*label_masks(label), complex(coeff)))
    for x, z, _ in out:
        if (x | z) >> num_qubits:
            raise ValueError("observable acts beyond the circuit's qubits")
    return out


def _is_observable(o: Any) -> bool:
    """One observable: a label, a dict, a SparsePauliOp-like object, or a
    sequence of term tuples ((label, coeff) or (x, z, coeff))."""
    if isinstance(o, (str, dict)) or hasattr(o, "paulis"):
        return True
    return isinstance(o, (list, tuple)) and len(o) > 0 and all(isinstance(t, tuple) for t in o)


def _observable_array(observables: Any) -> np.ndarray:
    """Observables (one, or nested sequences of them) as an object ndarray
    with one observable per element."""
    if _is_observable(observables):
        arr = np.empty((), object)
        arr[()] = observables
        return arr
    subs = [_observable_array(o) for o in observables]
    if not subs or any(s.shape != subs[0].shape for s in subs):
        raise ValueError("observables must form a regular array")
    arr = np.empty((len(subs),) + subs[0].shape, object)
    for i, sub in enumerate(subs):
        for idx in np.ndindex(*sub.shape):
            arr[(i,) + idx] = sub[idx]
    return arr


def parameter_slots(circ: Circuit) -> int:
    """Parameters the circuit's parameterised gates take, in op order."""
    return sum(NUM_PARAMS.get(oc, 0) for oc, *_ in circ.ops if oc not in (OP["unitary"], OP["measure"]))


def bind(circ: Circuit, values: Sequence[float]) -> Circuit:
    """The circuit with its parameterised gates' parameters taken, in op
    order, from `values` (the binding mb2_sweep_batch applies)."""
    values = list(values)
    if len(values) != parameter_slots(circ):
        raise ValueError(f"{len(values)} parameter values for {parameter_slots(circ)} slots")
    out = Circuit(circ.num_qubits, circ.num_clbits, circ.global_phase)
    k = 0
    for oc, qs, ps, m, cl in circ.ops:
        npar = 0 if oc in (OP["unitary"], OP["measure"]) else NUM_PARAMS.get(oc, 0)
        out.ops.append((oc, qs, tuple(float(v) for v in values[k:k + npar]) if npar else ps, m, cl))
        k += npar
    return out


class B200Estimator:
    """BaseEstimatorV2-shaped: ``run(pubs, precision=None)`` returns a list of
    results, one per pub: {"evs", "stds", "shape", "metadata"}.  A pub is
    (circuit, observables) or (circuit, observables, parameter_values) or
    (circuit, observables, parameter_values, precision)."""

    def __init__(self, ctx: Context | None = None, *, state_precision: int = _lib.C128,
                 default_precision: float = 0.0, seed: int | None = None, workers: int = 4):
        self.ctx = ctx if ctx is not None else Context(0)
        self.state_precision = state_precision
        self.default_precision = default_precision
        self.seed = seed
        self.workers = workers

    def run(self, pubs, *, precision: float | None = None) -> list[dict]:
        precision = self.default_precision if precision is None else precision
        seed = self.seed if self.seed is not None else secrets.randbits(63)
        pubs = [self._coerce(p, precision) for p in pubs]
        with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, self.workers)) as ex:
            return list(ex.map(lambda p: self._run_pub(p, seed), pubs))

    @staticmethod
    def _coerce(pub, precision):
        pub = tuple(pub)
        circ, observables = pub[0], pub[1]
        values = pub[2] if len(pub) > 2 else None
        prec = pub[3] if len(pub) > 3 and pub[3] is not None else precision
        return circ, _observable_array(observables), values, prec

    def _run_pub(self, pub, seed) -> dict:
        circ, obs, values, prec = pub
        n = circ.num_qubits
        terms_of = np.empty(obs.shape, object)
        for idx in np.ndindex(*obs.shape):
            terms_of[idx] = observable_terms(obs[idx], n)
        if values is None or parameter_slots(circ) == 0:
            evs = self._evs_one_state(circ, terms_of)
        else:
            evs = self._evs_bindings(circ, terms_of, np.asarray(values, np.float64))
        return {"evs": evs, "stds": np.zeros_like(evs), "shape": evs.shape,
                "metadata": {"target_precision": prec, "seed": seed, "state_precision": self.state_precision}}

    def _evs_one_state(self, circ, terms_of) -> np.ndarray:
        # The union of every observable's terms, read in one grouped pass.
        index: dict[tuple[int, int], int] = {}
        for idx in np.ndindex(*terms_of.shape):
            for x, z, _ in terms_of[idx]:
                index.setdefault((x, z), len(index))
        paulis = list(index)
        if self.state_precision == _lib.C64:
            paulis.append((0, 0))  # the norm, to renormalise in FP64
        st = DeviceState(self.ctx, circ.num_qubits, self.state_precision)
        try:
            st.init(circ.global_phase)
            st.apply_program(circ)
            vals = st.expectation(paulis)
        finally:
            st.free()
        norm = vals[-1].real if self.state_precision == _lib.C64 else 1.0
        evs = np.zeros(terms_of.shape, np.float64)
        for idx in np.ndindex(*terms_of.shape):
            evs[idx] = sum((c * vals[index[(x, z)]]).real for x, z, c in terms_of[idx]) / norm
        return evs

    def _evs_bindings(self, circ, terms_of, values) -> np.ndarray:
        slots = parameter_slots(circ)
        if values.shape[-1] != slots:
            raise ValueError(f"parameter values' last axis is {values.shape[-1]}, the circuit has {slots} slots")
        bshape = values.shape[:-1]
        flat = values.reshape(-1, slots)
        shape = np.broadcast_shapes(bshape, terms_of.shape)
        per_obs = {}
        batched = (_BATCH_MIN_QUBITS <= circ.num_qubits <= _BATCH_MAX_QUBITS and
                   all(len(terms_of[idx]) <= _lib.BATCH_MAX_TERMS for idx in np.ndindex(*terms_of.shape)))
        if batched:
            for idx in np.ndindex(*terms_of.shape):
                terms = terms_of[idx]
                # <P> is real for the Hermitian P = i^{|x&z|} X^x Z^z, so
                # Re(c <P>) = Re(c) <P>: mb2_sweep_batch's real weights.
                ws = [c.real for _, _, c in terms]
                paulis = [(x, z) for x, z, _ in terms]
                vals, _, _ = sweep_batch(self.ctx, circ, flat, paulis, ws, fuse_gates=True,
                                         precision=self.state_precision)
                per_obs[idx] = vals.reshape(bshape)
        else:  # beyond the batched sweep's sizes: one state per binding, all observables at once
            rows = [self._evs_one_state(bind(circ, v), terms_of) for v in flat]
            for idx in np.ndindex(*terms_of.shape):
                per_obs[idx] = np.array([r[idx] for r in rows]).reshape(bshape)
        evs = np.zeros(shape, np.float64)
        for idx in np.ndindex(*shape):
            b_idx = tuple(i if s > 1 else 0 for i, s in zip(idx[len(shape) - len(bshape):], bshape))
            o_idx = tuple(i if s > 1 else 0 for i, s in zip(idx[len(shape) - len(terms_of.shape):], terms_of.shape))
            evs[idx] = per_obs[o_idx][b_idx] if bshape else per_obs[o_idx]
        return evs


class B200Sampler:
    """BaseSamplerV2-shaped: ``run(pubs, shots=None)`` returns one result per
    pub: {"counts" (bitstring -> shots; for a parameterised pub an array of
    them over the bindings' shape), "shape", "metadata"}.  A pub is
    (circuit,), (circuit, parameter_values) or (circuit, parameter_values,
    shots); the circuit's measurements give the (qubit, clbit) pairs,
    last write wins.  Every pub and binding is one serving-loop request."""

    def __init__(self, ctx: Context | None = None, *, state_precision: int = _lib.C128,
                 default_shots: int = 1024, seed: int | None = None, budget_bytes: int = 0, slots: int = 0):
        from .serve import Server
        self.ctx = ctx if ctx is not None else Context(0)
        self.state_precision = state_precision
        self.default_shots = default_shots
        self.seed = seed
        self._server = Server(self.ctx, budget_bytes, slots)

    def close(self) -> None:
        self._server.close()

    def run(self, pubs, *, shots: int | None = None) -> list[dict]:
        shots = self.default_shots if shots is None else shots
        seed = self.seed if self.seed is not None else secrets.randbits(63)
        rng = np.random.default_rng(seed)
        jobs = []  # (pub index, binding index, ticket)
        meta = []
        for pi, pub in enumerate(pubs):
            pub = tuple(pub)
            circ = pub[0]
            values = pub[1] if len(pub) > 1 and pub[1] is not None else None
            s = int(pub[2]) if len(pub) > 2 and pub[2] is not None else shots
            targets = circ.measure_targets()
            if not targets:
                raise ValueError("a sampler pub's circuit has no measurements")
            width = max(c for _, c in targets) + 1
            if values is None or parameter_slots(circ) == 0:
                bshape, bound = (), [circ]
            else:
                values = np.asarray(values, np.float64)
                bshape = values.shape[:-1]
                bound = [bind(circ, v) for v in values.reshape(-1, values.shape[-1])]
            for bi, c in enumerate(bound):
                t = self._server.submit(c, "counts", shots=s, seed=int(rng.integers(0, 2 ** 63)), targets=targets,
                                        precision=self.state_precision)
                jobs.append((pi, bi, t))
            meta.append((bshape, width, s))
        done = {}
        while len(done) < len(jobs):
            for d in self._server.poll(200):
                if d["status"] != 0:
                    raise RuntimeError(f"sampler request failed with status {d['status']}")
                done[d["ticket"]] = d["counts"] or {}
        results = [None] * len(meta)
        for pi, (bshape, width, s) in enumerate(meta):
            tickets = [t for p, _, t in jobs if p == pi]
            as_bits = [{format(k, f"0{width}b"): v for k, v in sorted(done[t].items())} for t in tickets]
            if bshape:
                counts = np.empty(bshape, object)
                for i, idx in enumerate(np.ndindex(*bshape)):
                    counts[idx] = as_bits[i]
            else:
                counts = as_bits[0]
            results[pi] = {"counts": counts, "shape": bshape, "metadata": {"shots": s, "seed": seed}}
        return results
