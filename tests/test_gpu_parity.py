"""Parity of the sm_100a plain complex128 path with the CPU oracle, through
the C ABI.  Bitwise for every amplitude and for counts; expectation values
within 1e-12 absolute (a parallel FP64 reduction against the oracle's
sequential sum, the tolerance the reference's own CPU/CUDA differential test
uses, docs/adr/0014: worst 8.3e-13).  Modelled on the reference's
tests/api/cpu_cuda_differential_test.cpp and
tests/engines/dense/cuda_specialised_kernels_test.cpp."""
import numpy as np
import pytest

from menos_b200 import B200DenseEngine, DeviceState, EngineExecutionRequest, PauliTerm, workloads
from menos_b200.engine import C64 as MB2_C64, C128 as MB2_C128
from menos_b200._lib import MB2Error, ResourceExceeded
from menos_b200.circuit import OP, Circuit
from test_host import as_oracle_circuit
from test_oracle_pin import Y_CONVENTION, bits_equal, rand_state, rand_unitary, random_circuit

pytestmark = pytest.mark.gpu

EXP_TOL = 1e-12
NAMES_1Q = ["x", "y", "z", "h", "s", "sdg", "t", "tdg", "sx", "sxdg", "rx", "ry", "rz", "p", "u"]
NAMES_2Q = ["cx", "cz", "swap", "cp", "rzz"]
NPAR = {"rx": 1, "ry": 1, "rz": 1, "p": 1, "cp": 1, "rzz": 1, "u": 3}


def dev_state(ctx, amps):
    n = int(np.log2(amps.size))
    st = DeviceState(ctx, n)
    st.copy_in(amps)
    return st


@pytest.mark.parametrize("phase", [0.0, -0.0, 1.0, -2.5, np.pi, 1e-300])
def test_init_global_phase(ctx, oracle, phase):
    for n in (1, 5, 12):
        st = DeviceState(ctx, n)
        st.init(phase)
        assert bits_equal(st.copy_out(), oracle.initialize(n, phase))


@pytest.mark.parametrize("n", [3, 8, 13])
def test_every_named_gate_on_every_operand(ctx, oracle, n):
    rng = np.random.default_rng(n)
    s0 = rand_state(n, rng)
    st = dev_state(ctx, s0)
    expect = s0.copy()
    for name in NAMES_1Q + NAMES_2Q + ["ccx"]:
        nq = 3 if name == "ccx" else (2 if name in NAMES_2Q else 1)
        if nq > n:
            continue
        m = oracle.gate_matrix(OP[name], rng.uniform(-7, 7, size=3)[:NPAR.get(name, 0)])
        if nq == 1:
            placements = [[q] for q in range(n)]
        elif nq == 2:
            placements = [[a, b] for a in range(n) for b in range(n) if a != b]
        else:
            placements = [list(rng.permutation(n)[:3]) for _ in range(6)]
        for qs in placements:
            oracle.apply_generic(expect, m, qs)
            st.apply_matrix(m, qs)
    assert bits_equal(st.copy_out(), expect)


def test_generic_kernel_every_width(ctx, oracle):
    rng = np.random.default_rng(5)
    n = 11
    s0 = rand_state(n, rng)
    a = dev_state(ctx, s0)
    b = dev_state(ctx, s0)
    expect = s0.copy()
    for k in range(1, 7):
        for _ in range(4):
            ops = list(rng.permutation(n)[:k])
            u = rand_unitary(k, rng)
            oracle.apply_generic(expect, u, ops)
            a.apply_matrix(u, ops)
            b.apply_matrix(u, ops, generic=True)
    assert bits_equal(a.copy_out(), expect)
    assert bits_equal(b.copy_out(), expect)


def test_signed_zeros_diagonals_and_permutations(ctx, oracle):
    # Mirrors specialised_kernels_test.cpp:82-102: -0.0 components in the
    # state, and matrices whose entries are signed zeros and +-1.
    n = 6
    rng = np.random.default_rng(1)
    s0 = rand_state(n, rng)
    s0.real[::3] = -0.0
    s0.imag[1::4] = -0.0
    s0[7] = complex(-0.0, -0.0)
    mats = [
        ([2], np.array([[1, 0], [0, -1]], np.complex128)),
        ([1], np.array([[complex(0.0, -0.0), 1], [1, complex(-0.0, 0.0)]], np.complex128)),
        ([0, 4], oracle.gate_matrix(OP["cz"])),
        ([5, 0], oracle.gate_matrix(OP["swap"])),
        ([3, 2], oracle.gate_matrix(OP["cx"])),
        ([1, 3, 5], np.diag(np.exp(1j * rng.uniform(0, 6, 8)))),
        ([4], np.array([[complex(-1, -0.0), 0], [0, complex(1, 0.0)]], np.complex128)),
    ]
    for generic in (False, True):
        st = dev_state(ctx, s0)
        expect = s0.copy()
        for qs, m in mats:
            oracle.apply_generic(expect, m, qs)
            st.apply_matrix(m, qs, generic=generic)
        assert bits_equal(st.copy_out(), expect), generic


@pytest.mark.parametrize("tile", [0, 4, 6, 9, 12])
def test_tiled_program_bitwise(ctx, oracle, tile):
    rng = np.random.default_rng(100 + tile)
    for n in (1, 2, 3, 4, 5, 7, 10, 12, 14):
        for fuse in (True, False):
            c = random_circuit(n, 90, rng)
            st = DeviceState(ctx, n)
            st.init(c.global_phase)
            st.apply_program(c, fuse_gates=fuse, tile_qubits=tile)
            expect = oracle.run(as_oracle_circuit(c), fuse_gates=fuse)
            assert bits_equal(st.copy_out(), expect), (n, fuse, tile)


def test_long_program_splits_passes(ctx, oracle):
    # More blocks than one pass may hold on a state that fits a single tile.
    rng = np.random.default_rng(8)
    n = 10
    c = random_circuit(n, 800, rng, unitaries=False)
    st = DeviceState(ctx, n)
    st.init(c.global_phase)
    stats = st.apply_program(c, fuse_gates=False)
    assert stats.passes >= 3
    assert bits_equal(st.copy_out(), oracle.run(as_oracle_circuit(c), fuse_gates=False))


def test_per_gate_sweep_bitwise(ctx, oracle):
    rng = np.random.default_rng(77)
    for n in (3, 9, 13):
        c = random_circuit(n, 60, rng)
        st = DeviceState(ctx, n)
        st.init(c.global_phase)
        st.apply_program(c, fuse_gates=True, per_gate=True)
        assert bits_equal(st.copy_out(), oracle.run(as_oracle_circuit(c), fuse_gates=True))


def test_brick_and_qft_against_reference(ctx, oracle, ref):
    # The benchmark's own gate families at 16 qubits, against the reference engine.
    c = workloads.brick(16, 12, 3)
    workloads.qft(16, c)
    oc = as_oracle_circuit(c)
    expect = ref.run(oc, fuse_gates=True)["statevector"]
    for tile in (0, 8, 12):
        st = DeviceState(ctx, 16)
        st.init(0.0)
        st.apply_program(c, tile_qubits=tile)
        assert bits_equal(st.copy_out(), expect), tile


def test_config_c1_statevector_and_counts(ctx, ref):
    # 20 qubits, 20 brick layers: statevector + 4096 shots, as the reference engine runs it.
    c = workloads.config_c1()
    oc = as_oracle_circuit(c)
    targets = [(q, q) for q in range(20)]
    r = ref.run(oc, fuse_gates=True, statevector=True, shots=4096, seed=1234, targets=targets, width=20)
    eng = B200DenseEngine()
    res = eng.execute(EngineExecutionRequest(num_qubits=20, operations=c, want_statevector=True, want_counts=True,
                                             shots=4096, seed=1234, measure_targets=targets, bitstring_width=20))
    assert bits_equal(res.statevector, r["statevector"])
    assert res.counts == r["counts"]


def test_expectation_within_tolerance(ctx, oracle):
    rng = np.random.default_rng(9)
    for n in (1, 2, 6, 11, 15):
        s = rand_state(n, rng)
        st = dev_state(ctx, s)
        terms = [(0, 0)] + [(int(rng.integers(0, 1 << n)), int(rng.integers(0, 1 << n))) for _ in range(24)]
        got = st.expectation(terms)
        for (x, z), g in zip(terms, got):
            e = oracle.expectation(s, x, z)
            assert abs(g - e) <= EXP_TOL, (n, x, z, g, e)
        assert abs(st.norm() - 1.0) <= EXP_TOL


def test_expectation_y_convention(ctx):
    # Qiskit's Y = i X Z: <+i|Y|+i> = 1 (reference dense_engine_test.cpp:279-330).
    st = DeviceState(ctx, 1)
    st.copy_in(np.array([1, 1j], np.complex128) / np.sqrt(2))
    v = st.expectation([(1, 1), (1, 0), (0, 1)])
    assert abs(v[0] - 1.0) < 1e-15 and abs(v[1]) < 1e-15 and abs(v[2]) < 1e-15
    # The reference's circuits for the same convention, through the sweep.
    for n, gates, terms in Y_CONVENTION:
        c = Circuit(n)
        for name, qs in gates:
            c.gate(name, qs)
        st = DeviceState(ctx, n)
        st.init(0.0)
        st.apply_program(c)
        got = st.expectation([(x, z) for x, z, _ in terms])
        for (x, z, want), g in zip(terms, got):
            assert abs(g - want) <= EXP_TOL, (n, x, z, g)


def test_sampling_identical_counts(ctx, oracle):
    rng = np.random.default_rng(4)
    for n in (1, 3, 10, 16):
        s = rand_state(n, rng)
        st = dev_state(ctx, s)
        for shots, seed in [(1, 0), (20, 42), (4096, 7), (100000, 2 ** 40 + 3)]:
            t = [(q, q) for q in range(n)]
            assert st.sample(shots, seed, t) == oracle.sample(s, shots, seed, t), (n, shots)
        t = [(0, 2), (n - 1, 0)]
        assert st.sample(3000, 5, t) == oracle.sample(s, 3000, 5, t)


def test_sampling_golden_plus_state(ctx):
    st = DeviceState(ctx, 1)
    st.copy_in(np.array([1, 1], np.complex128) / np.sqrt(2.0))
    assert st.sample(20, 42, [(0, 0)]) == {0: 9, 1: 11}
    # tests/engines/dense/sample_test.cpp:39-83: zero shots give no counts;
    # basis bits reach clbits through the targets (|q1=1, q0=0>, q0 -> c1,
    # q1 -> c0: outcome 1).
    assert st.sample(0, 1, [(0, 0)]) == {}
    st2 = DeviceState(ctx, 2)
    st2.copy_in(np.array([0, 0, 1, 0], np.complex128))
    assert st2.sample(10, 1, [(0, 1), (1, 0)]) == {1: 10}


def test_engine_execute_matches_reference(ctx, ref):
    rng = np.random.default_rng(31)
    for n in (2, 7, 12):
        c = random_circuit(n, 50, rng)
        oc = as_oracle_circuit(c)
        paulis = [(int(rng.integers(0, 1 << n)), int(rng.integers(0, 1 << n))) for _ in range(8)]
        targets = [(q, q) for q in range(n)]
        r = ref.run(oc, statevector=True, shots=2000, seed=5, targets=targets, width=n, paulis=paulis)
        eng = B200DenseEngine()
        res = eng.execute(EngineExecutionRequest(
            num_qubits=n, operations=c, global_phase=c.global_phase, want_statevector=True, want_counts=True,
            want_expectation=True, shots=2000, seed=5, measure_targets=targets, bitstring_width=n,
            observable=[PauliTerm(x, z) for x, z in paulis]))
        assert bits_equal(res.statevector, r["statevector"])
        assert res.counts == r["counts"]
        assert np.max(np.abs(res.expectation_terms - r["terms"])) <= EXP_TOL


def test_budget_and_invalid_arguments(ctx):
    with pytest.raises(ResourceExceeded):
        DeviceState(ctx, 20, budget_bytes=(16 << 20) - 1)
    st = DeviceState(ctx, 4)
    with pytest.raises(MB2Error):
        st.apply_matrix(np.eye(2), [4])
    with pytest.raises(MB2Error):
        st.apply_matrix(np.eye(4), [1, 1])
    with pytest.raises(MB2Error):
        st.expectation([(1 << 5, 0)])
    c = Circuit(4).gate("h", [7])
    with pytest.raises(MB2Error):
        st.apply_program(c)


def test_large_state_tiled_equals_per_gate(ctx):
    # Size-independent property at 26 qubits (1 GiB): the tiled sweep and the
    # one-launch-per-block sweep agree bitwise, and the norm stays 1.
    n = 26
    c = workloads.brick(n, 6, 11)
    workloads.qft(n, c)
    a = DeviceState(ctx, n)
    a.init(0.0)
    a.apply_program(c)
    b = DeviceState(ctx, n)
    b.init(0.0)
    b.apply_program(c, per_gate=True)
    xa, xb = a.copy_out(), b.copy_out()
    assert bits_equal(xa, xb)
    assert abs(a.norm() - 1.0) < 1e-10


def test_autotune_and_time_model(ctx):
    # The autotuner picks widths it measured and feeds a time model that
    # predicts a brick sweep within a factor of two; the tuned widths stay
    # bitwise (the plain path does not depend on the tile width).
    t = ctx.autotune()
    assert t["tile_qubits"] in (10, 11, 12) and t["tile_qubits_c64"] in (12, 13)
    assert t["probe_qubits"] == 24 and t["pass_s_per_amp"] > 0 and t["dense1_s_per_amp"] > 0
    assert ctx.tuning()["tile_qubits"] == t["tile_qubits"]
    import time
    n = 26
    for c, precision in ((workloads.brick(n, 20, 3), MB2_C128), (workloads.qft(n), MB2_C128),
                         (workloads.brick(n, 20, 3), MB2_C64)):
        st = DeviceState(ctx, n, precision=precision)
        st.init(0.0)
        st.apply_program(c)
        st.synchronize()
        t0 = time.perf_counter()
        st.apply_program(c)
        st.synchronize()
        measured = time.perf_counter() - t0
        est = ctx.estimate_time(c, precision=precision)
        assert 0.5 * measured <= est <= 2.0 * measured, (est, measured, precision)
    small = workloads.brick(14, 6, 4)
    a = DeviceState(ctx, 14)
    a.init(0.0)
    a.apply_program(small)
    b = DeviceState(ctx, 14)
    b.init(0.0)
    b.apply_program(small, tile_qubits=11)
    assert bits_equal(a.copy_out(), b.copy_out())
