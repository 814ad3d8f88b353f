"""The trajectory engine (the reference's TrajectoryEngine,
src/engines/trajectory/trajectory_engine.cpp).

CPU: a Python restatement of the reference's algorithm -- SplitMix64
trajectory seeds, one common::Rng uniform per channel and one word per shot,
branch by cumulative Re Tr(K^dagger K rho_q), the reference's own
apply_matrix for gates and branches, the sequential norm -- reproduces the
reference engine's term means bit for bit, and its means approach the exact
density-matrix values as the trajectory count grows.

GPU: mb2_trajectories gives the reference engine's counts exactly and its
term means within 1e-12 (each trajectory's state is the reference's; the
per-trajectory expectations are this engine's grouped reductions).
"""
import math

import numpy as np
import pytest

import pyoracle
from test_dm import noisy_circuit

MASK64 = (1 << 64) - 1


def trajectory_seed(seed, t):
    z = (seed + (t + 1) * 0x9E3779B97F4A7C15) & MASK64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return z ^ (z >> 31)


def restated_trajectories(ref, circ, count, seed, paulis):
    """The reference's trajectory loop restated over its own kernels."""
    n = circ.num_qubits
    sums = np.zeros(len(paulis), np.complex128)
    for t in range(count):
        draws = iter(ref.uniforms(trajectory_seed(seed, t), 64))
        psi = np.zeros(1 << n, np.complex128)
        psi[0] = 1.0
        for oc, qs, ps, m, _cl in circ.ops:
            if oc == pyoracle.OP["measure"]:
                continue
            if oc != pyoracle.OP["channel"]:
                ref.apply_matrix(psi, m if m is not None else ref.gate_matrix(oc, ps), list(qs), threads=1)
                continue
            k = len(qs)
            dim = 1 << k
            rho = np.zeros((dim, dim), np.complex128)
            mask = sum(1 << q for q in qs)
            for base in range(1 << n):
                if base & mask:
                    continue
                sl = [psi[base | sum(1 << qs[j] for j in range(k) if (a >> j) & 1)] for a in range(dim)]
                for r in range(dim):
                    for c in range(dim):
                        rho[r, c] += sl[r] * np.conj(sl[c])
            u = next(draws)
            cum, branch, last = 0.0, None, None
            for i, kmat in enumerate(m):
                prod = kmat.conj().T @ kmat
                p = sum((prod[a, b] * rho[b, a]).real for a in range(dim) for b in range(dim))
                if p > 0.0:
                    last = i
                    cum += p
                    if u < cum:
                        branch = i
                        break
            branch = last if branch is None else branch
            ref.apply_matrix(psi, m[branch], list(qs), threads=1)
            norm_sq = 0.0
            for a in psi:
                norm_sq += a.real * a.real + a.imag * a.imag
            psi *= 1.0 / math.sqrt(norm_sq)
        for i, (x, z) in enumerate(paulis):
            sums[i] += ref.expectation(psi, x, z)
    # std::complex /= double divides each part (trajectory_engine.cpp:480-483).
    out = np.empty_like(sums)
    out.real = sums.real / count
    out.imag = sums.imag / count
    return out


def pure_noise_circuit(n, depth, seed, widest=2):
    c, _ = noisy_circuit(n, depth, np.random.default_rng(seed), widest=widest)
    return c


def test_trajectory_seed_is_the_matching_splitmix64_output():
    """tests/engines/trajectory/trajectory_engine_test.cpp:67-73: trajectory
    t's seed is output t of one SplitMix64 stream seeded with the job's
    seed (state += 0x9E3779B97F4A7C15, then the published output mix)."""
    state = 0xDEADBEEF
    for t in range(8):
        state = (state + 0x9E3779B97F4A7C15) & MASK64
        z = ((state ^ (state >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        assert trajectory_seed(0xDEADBEEF, t) == z ^ (z >> 31)


def test_restatement_is_bitwise_the_reference_engine(ref):
    n = 5
    c = pure_noise_circuit(n, 30, 1)
    paulis = [(0, 1), (3, 0), (5, 5), (0, 0)]
    r = ref.run_trajectories(c, 12, 99, paulis=paulis)
    mine = restated_trajectories(ref, c, 12, 99, paulis)
    assert np.array_equal(mine.view(np.uint64), r["terms"].view(np.uint64))


def test_reference_trajectories_approach_the_density_matrix(ref):
    n = 4
    c = pure_noise_circuit(n, 24, 2)
    paulis = [(int(x), int(z)) for x, z in np.random.default_rng(3).integers(0, 1 << n, size=(6, 2))]
    exact = ref.run_dm(c, threads=1, paulis=paulis)["terms"]
    r = ref.run_trajectories(c, 3000, 5, paulis=paulis)
    # Each term's mean within 5 standard errors (|<P>| <= 1: s <= 1/sqrt(N)).
    assert np.max(np.abs(r["terms"] - exact)) < 5 / math.sqrt(3000)
    assert r["standard_error"] > 0


@pytest.mark.gpu
@pytest.mark.parametrize("n", [3, 8, 13])
def test_device_trajectories_match_the_reference(ctx, ref, n):
    from menos_b200 import Circuit
    from menos_b200.engine import trajectories
    c = pure_noise_circuit(n, 40, 10 + n, widest=3)
    d = Circuit(n)
    d.ops = list(c.ops)
    rng = np.random.default_rng(n)
    paulis = [(int(x), int(z)) for x, z in rng.integers(0, 1 << n, size=(8, 2))] + [(0, 0)]
    coefs = rng.normal(size=len(paulis)) + 1j * rng.normal(size=len(paulis))
    targets = [(q, n - 1 - q) for q in range(n)]
    count, shots = 96, 80
    got = trajectories(ctx, d, count, 2026, paulis, coefs, shots, targets)
    want = ref.run_trajectories(c, count, 2026, paulis=paulis, coefs=coefs, shots=shots, targets=targets)
    assert got["counts"].to_dict() == want["counts"]
    assert np.max(np.abs(got["terms"] - want["terms"])) < 1e-12
    assert abs(got["standard_error"] - want["standard_error"]) <= 1e-9 * max(1.0, want["standard_error"])


@pytest.mark.gpu
@pytest.mark.parametrize("n", [2, 7])
def test_device_trajectory_readout_counts_are_the_reference(ctx, ref, n):
    """Readout errors on the measurements: after each shot's word, one per
    readout-errored target (trajectory_engine.cpp:465-471)."""
    from menos_b200 import Circuit
    from menos_b200.engine import trajectories
    from test_dm import with_readout_measures
    c = pure_noise_circuit(n, 30, 40 + n, widest=2)
    d = Circuit(n)
    d.ops = list(c.ops)
    targets = with_readout_measures([c, d], n, np.random.default_rng(n))
    count = shots = 160
    got = trajectories(ctx, d, count, 77, shots=shots, targets=targets)
    want = ref.run_trajectories(c, count, 77, shots=shots, targets=targets)
    assert got["counts"].to_dict() == want["counts"]


@pytest.mark.gpu
def test_device_exact_norm_is_the_sequential_sum(ctx):
    from menos_b200 import DeviceState, workloads
    n = 18
    st = DeviceState(ctx, n)
    st.init(0.3)
    st.apply_program(workloads.brick(n, 6, 1))
    psi = st.copy_out()
    seq = 0.0
    for a in psi.tolist():
        seq += a.real * a.real + a.imag * a.imag
    assert st.norm_exact() == seq
