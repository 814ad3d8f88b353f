"""The batched parameter sweep against single runs: every binding's state is
bitwise the state the reference engine computes for that binding alone, and
<H> agrees within the expectation tolerance."""
import numpy as np
import pytest

from menos_b200 import workloads
from menos_b200.engine import sweep_batch
from test_host import as_oracle_circuit
from test_oracle_pin import bits_equal

pytestmark = pytest.mark.gpu


def bound_circuit(n, layers, row):
    c = workloads.hea(n, layers, 0)
    k = 0
    ops = []
    for oc, qs, ps, m, cl in c.ops:
        if ps:
            ps = tuple(row[k:k + len(ps)])
            k += len(ps)
        ops.append((oc, qs, ps, m, cl))
    c.ops = ops
    return c


@pytest.mark.parametrize("fuse", [False, True])
def test_batch_matches_single_runs(ctx, ref, fuse):
    n, layers, B = 10, 4, 13
    rows = workloads.hea_bindings(n, layers, B, 99)
    paulis = workloads.pauli_strings(n, 32, 5)
    coefs = workloads.weights(32, 6)
    vals, states, stats = sweep_batch(ctx, workloads.hea(n, layers, 0), rows, paulis, coefs, fuse_gates=fuse,
                                      want_states=True)
    assert stats.parametric_blocks > 0
    for b in range(B):
        c = as_oracle_circuit(bound_circuit(n, layers, rows[b]))
        r = ref.run(c, fuse_gates=fuse, statevector=True, paulis=paulis)
        assert bits_equal(states[b], r["statevector"]), b
        h = sum(w * t for w, t in zip(coefs, r["terms"]))
        assert abs(vals[b] - h.real) <= 1e-12 * max(1.0, sum(abs(w) for w in coefs)), (b, vals[b], h)


def test_batch_hea16_subset(ctx, ref):
    # The benchmark's shape (16 qubits, 8 layers, 32 terms) on a few bindings.
    n, layers, B = 16, 8, 9
    rows = workloads.hea_bindings(n, layers, B, 2026)
    paulis = workloads.pauli_strings(n, 32, 7)
    coefs = workloads.weights(32, 8)
    vals, states, stats = sweep_batch(ctx, workloads.hea(n, layers, 0), rows, paulis, coefs, want_states=True)
    for b in (0, 4, 8):
        c = as_oracle_circuit(bound_circuit(n, layers, rows[b]))
        r = ref.run(c, fuse_gates=False, statevector=True, paulis=paulis)
        assert bits_equal(states[b], r["statevector"])
        h = sum(w * t for w, t in zip(coefs, r["terms"]))
        assert abs(vals[b] - h.real) <= 1e-11


def test_batch_complex64_within_tolerance(ctx):
    # The complex64 batch against the complex128 one (itself bitwise the
    # reference): <H> within the precision path's 1e-6, states within 1e-5.
    from menos_b200._lib import C64
    n, layers, B = 16, 8, 24
    rows = workloads.hea_bindings(n, layers, B, 31)
    paulis = workloads.pauli_strings(n, 32, 32)
    coefs = workloads.weights(32, 33)
    circ = workloads.hea(n, layers, 0)
    hi, s_hi, _ = sweep_batch(ctx, circ, rows, paulis, coefs, want_states=True)
    lo, s_lo, stats = sweep_batch(ctx, circ, rows, paulis, coefs, want_states=True, precision=C64)
    assert stats.parametric_blocks > 0
    assert np.max(np.abs(lo - hi)) <= 1e-6
    assert np.max(np.abs(s_lo - s_hi)) <= 1e-5


@pytest.mark.parametrize("n", [11, 12])
def test_batch_grouped_expectation_many_bindings(ctx, ref, n):
    # More bindings than the grouped reduction has binding lanes (each lane
    # takes several bindings in turn), at the smallest grouped sizes (one and
    # two CTAs per binding).
    layers, B = 3, 333
    rows = workloads.hea_bindings(n, layers, B, 400 + n)
    paulis = workloads.pauli_strings(n, 32, 401 + n)
    coefs = workloads.weights(32, 402 + n)
    vals, _, _ = sweep_batch(ctx, workloads.hea(n, layers, 0), rows, paulis, coefs)
    for b in (0, 1, 147, 295, 296, 297, 332):
        c = as_oracle_circuit(bound_circuit(n, layers, rows[b]))
        r = ref.run(c, fuse_gates=True, paulis=paulis)
        h = sum(w * t for w, t in zip(coefs, r["terms"]))
        assert abs(vals[b] - h.real) <= 1e-11, (b, vals[b], h)


@pytest.mark.parametrize("fuse", [False, True])
def test_batch_binding_at_angle_zero_bitwise(ctx, ref, fuse):
    # RY(0) and RZ(0) are diagonal (the identity) for one binding only: that
    # binding still runs the dense path the others need, and its state is
    # bitwise the reference's, whose dispatch takes the diagonal kernel.
    n, layers, B = 10, 3, 4
    rows = workloads.hea_bindings(n, layers, B, 123)
    rows[1][0] = 0.0          # RY(0) on qubit 0, first layer
    rows[1][3] = 0.0          # RZ(0) on qubit 1
    rows[2] = [0.0] * len(rows[2])
    paulis = workloads.pauli_strings(n, 8, 5)
    coefs = workloads.weights(8, 6)
    vals, states, _ = sweep_batch(ctx, workloads.hea(n, layers, 0), rows, paulis, coefs, fuse_gates=fuse,
                                  want_states=True)
    for b in range(B):
        c = as_oracle_circuit(bound_circuit(n, layers, rows[b]))
        r = ref.run(c, fuse_gates=fuse, statevector=True)
        assert bits_equal(states[b], r["statevector"]), b
