"""The complex64 tensor-core path (tcgen05 kind::f16, split-FP16 operands,
FP32 accumulation) on the GPU.

* The tensor-core step alone (mb2_debug_tc_probe): 256 rows of 16 complex
  amplitudes times a 16x16 complex matrix equal the FP64 product within the
  split's precision (about 2^-21 of the largest amplitude), for random
  unitaries, the identity and a permutation -- which pins the tensor-memory
  and shared-memory operand layouts.
* Whole sweeps: the tensor-core passes against the complex128 path (itself
  bitwise the reference) and against the FP32 SIMT passes, on every circuit
  family, at 12- and 13-qubit tiles: amplitudes within 1e-6 and Pauli
  expectations within 1e-6 (the precision path's bar)."""
import numpy as np
import pytest

from menos_b200 import DeviceState, workloads
from menos_b200._lib import C64
from test_tc_plan import CIRCUITS

pytestmark = pytest.mark.gpu


def rand_unitary(rng, d=16):
    m = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
    q, r = np.linalg.qr(m)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def test_tc_probe_matches_fp64_product(ctx):
    rng = np.random.default_rng(1)
    rows = (rng.standard_normal((256, 16)) + 1j * rng.standard_normal((256, 16))).astype(np.complex64)
    exact_in = rows.astype(np.complex128)
    for u in (rand_unitary(rng), rand_unitary(rng), np.eye(16), np.eye(16)[rng.permutation(16)],
              np.diag(np.exp(1j * rng.uniform(0, 2 * np.pi, 16)))):
        got = ctx.tc_probe(rows, u).astype(np.complex128)
        expect = exact_in @ u.T
        scale = np.max(np.abs(exact_in))
        err = np.max(np.abs(got - expect)) / scale
        assert err <= 4e-6, err


def test_tc_probe_row_and_column_placement(ctx):
    # One nonzero amplitude per row, a matrix with one nonzero per row: every
    # output lands where the layout says, exactly (every value is exact in FP16).
    rows = np.zeros((256, 16), np.complex64)
    for r in range(256):
        rows[r, r % 16] = (r + 1) + 0.5j * (r % 7)
    perm = np.roll(np.arange(16), 3)
    u = np.zeros((16, 16), np.complex128)
    u[np.arange(16), perm] = 1j
    got = ctx.tc_probe(rows, u)
    expect = (rows.astype(np.complex128) @ u.T).astype(np.complex64)
    assert np.array_equal(got, expect)


def c64_state(ctx, circ, kernel, tile):
    st = DeviceState(ctx, circ.num_qubits, precision=C64)
    st.init(circ.global_phase)
    stats = st.apply_program(circ, tile_qubits=tile, c64_kernel=kernel)
    return st, stats


@pytest.mark.parametrize("name", sorted(CIRCUITS))
@pytest.mark.parametrize("n,tile", [(14, 12), (15, 13), (18, 12), (18, 13)])
def test_tc_sweep_against_complex128(ctx, name, n, tile):
    circ = CIRCUITS[name](n)
    hi = DeviceState(ctx, n)
    hi.init(circ.global_phase)
    hi.apply_program(circ)
    hi_amps = hi.copy_out()
    paulis = workloads.pauli_strings(n, 16, n)
    hi_terms = hi.expectation(paulis)
    st, _ = c64_state(ctx, circ, "tensor", tile)
    amps = st.copy_out().astype(np.complex128)
    assert np.max(np.abs(amps - hi_amps)) <= 1e-6
    assert np.max(np.abs(st.expectation(paulis) - hi_terms)) <= 1e-6
    simt, _ = c64_state(ctx, circ, "simt", tile)
    assert np.max(np.abs(simt.copy_out().astype(np.complex128) - amps)) <= 1e-6


def test_tc_split_passes_on_a_small_state(ctx):
    # One tile holds the whole state: passes carry many phases and are split
    # at the shared-memory limit; the state is still the complex128 one.
    circ = workloads.brick(12, 40, 9)
    hi = DeviceState(ctx, 12)
    hi.init(0.0)
    hi.apply_program(circ)
    st, stats = c64_state(ctx, circ, "tensor", 12)
    assert np.max(np.abs(st.copy_out().astype(np.complex128) - hi.copy_out())) <= 1e-6
