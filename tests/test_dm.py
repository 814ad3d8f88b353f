"""The density-matrix path (the reference's DensityMatrixEngine,
src/engines/density_matrix/density_matrix_engine.cpp).

CPU: the reference engine itself (oracle/_ref) against a numpy restatement
of rho -> U rho U^dagger and rho -> sum_K K rho K^dagger, so the checker is
pinned before the device is compared with it.

GPU: the device rho is bitwise the reference's operation sequence (each gate
as apply_matrix with U on the row qubits then conj(U) on the column qubits,
each channel as apply_matrix with its superoperator), Pauli traces agree with
the reference engine within 1e-12 and its counts are identical.
"""
import numpy as np
import pytest

from test_oracle_pin import random_circuit

import pyoracle


def depolarizing(p):
    i2 = np.eye(2)
    x = np.array([[0, 1], [1, 0]])
    y = np.array([[0, -1j], [1j, 0]])
    z = np.diag([1, -1])
    return np.stack([np.sqrt(1 - 3 * p / 4) * i2] + [np.sqrt(p / 4) * m for m in (x, y, z)]).astype(np.complex128)


def amplitude_damping(g):
    return np.array([[[1, 0], [0, np.sqrt(1 - g)]], [[0, np.sqrt(g)], [0, 0]]], np.complex128)


def random_kraus(k, count, rng):
    """count Kraus operators on k qubits: blocks of a random isometry."""
    dim = 1 << k
    a = rng.normal(size=(count * dim, dim)) + 1j * rng.normal(size=(count * dim, dim))
    q, _ = np.linalg.qr(a)
    return np.ascontiguousarray(q.reshape(count, dim, dim))


def noisy_circuit(n, depth, rng, widest=3):
    """Gates of the dense path's random circuit with channels of up to
    `widest` qubits between them, as the oracle's circuit and the
    package's."""
    from menos_b200 import Circuit
    base = random_circuit(n, depth, rng)
    c = pyoracle.Circuit(n)
    d = Circuit(n)
    for i, (oc, qs, ps, m, cl) in enumerate(base.ops):
        c.ops.append((oc, qs, ps, m, cl))
        d.ops.append((oc, qs, ps, m, cl))
        if i % 4 == 3:
            kind = rng.integers(0, 3)
            if kind == 0:
                q, kr = (int(rng.integers(0, n)),), depolarizing(float(rng.uniform(0.01, 0.2)))
            elif kind == 1:
                q, kr = (int(rng.integers(0, n)),), amplitude_damping(float(rng.uniform(0.05, 0.5)))
            else:
                k = min(n, int(rng.integers(1, widest + 1)))
                q = tuple(int(v) for v in rng.choice(n, size=k, replace=False))
                kr = random_kraus(k, int(rng.integers(1, 4)), rng)
            c.channel(q, kr)
            d.channel(q, kr)
    return c, d


def apply_op(vec, nq, m, qubits):
    """numpy: matrix m on the given qubits of a 2^nq vector (bit j of m's
    index is qubits[j])."""
    k = len(qubits)
    t = vec.reshape([2] * nq)
    axes = [nq - 1 - q for q in qubits][::-1]
    mt = m.reshape([2] * (2 * k))
    out = np.tensordot(mt, t, axes=(list(range(k, 2 * k)), axes))
    rest = [a for a in range(nq) if a not in axes]
    perm = np.argsort(axes + rest)
    return np.transpose(out, perm).reshape(-1)


def numpy_rho(circ, gate_matrix):
    """rho = |0><0| evolved by the circuit, as a (2^n, 2^n) array."""
    n = circ.num_qubits
    dim = 1 << n
    rho = np.zeros((dim, dim), np.complex128)
    rho[0, 0] = 1.0
    for oc, qs, ps, m, _cl in circ.ops:
        if oc == pyoracle.OP["measure"]:
            continue
        if oc == pyoracle.OP["channel"]:
            mats = list(m)
        else:
            mats = [m if m is not None else gate_matrix(oc, ps)]
        new = np.zeros_like(rho)
        for kmat in mats:
            t = np.stack([apply_op(rho[:, col], n, kmat, qs) for col in range(dim)], axis=1)
            t = np.stack([apply_op(t[row, :].conj(), n, kmat, qs).conj() for row in range(dim)], axis=0)
            new += t
        rho = new
    return rho


def pauli_matrix(n, x, z):
    dim = 1 << n
    p = np.zeros((dim, dim), np.complex128)
    ph = 1j ** (bin(x & z).count("1") % 4)
    for c in range(dim):
        p[c ^ x, c] = ph * (-1) ** (bin(c & z).count("1") % 2)
    return p


def superoperator(kraus):
    """sum over K (in order) of K[r, r2] conj(K[c, c2]) at row r | c << k,
    column r2 | c2 << k (density_matrix_engine.cpp:78-100), each product
    formed as std::complex does it -- (ac - bd, ad + bc), every operation
    rounded on its own -- so the sum has the reference's bits."""
    dim = kraus.shape[1]
    sre = np.zeros((dim, dim, dim, dim))
    sim = np.zeros((dim, dim, dim, dim))
    for kmat in kraus:
        ar, ai = kmat.real[None, :, None, :], kmat.imag[None, :, None, :]      # K[r, r2]
        br, bi = kmat.real[:, None, :, None], -kmat.imag[:, None, :, None]     # conj(K[c, c2])
        sre = sre + (ar * br - ai * bi)
        sim = sim + (ar * bi + ai * br)
    out = np.empty((dim * dim, dim * dim), np.complex128)
    out.real = sre.reshape(dim * dim, dim * dim)
    out.imag = sim.reshape(dim * dim, dim * dim)
    return out


def reference_rho_vector(ref, circ):
    """The reference engine's operation sequence (apply_unitary /
    apply_channel, density_matrix_engine.cpp:68-118) through its own
    apply_matrix on the 2n-qubit vector, with the superoperator summed in its
    order: the bits the reference's rho holds."""
    n = circ.num_qubits
    vec = np.zeros(1 << (2 * n), np.complex128)
    vec[0] = 1.0
    for oc, qs, ps, m, _cl in circ.ops:
        if oc == pyoracle.OP["measure"]:
            continue
        cols = [q + n for q in qs]
        if oc == pyoracle.OP["channel"]:
            ref.apply_matrix(vec, superoperator(m), list(qs) + cols, threads=1)
        else:
            u = m if m is not None else ref.gate_matrix(oc, ps)
            ref.apply_matrix(vec, u, list(qs), threads=1)
            ref.apply_matrix(vec, np.conj(u), cols, threads=1)
    return vec


@pytest.mark.parametrize("n", [1, 2, 3, 5])
def test_reference_dm_engine_matches_numpy(ref, n):
    rng = np.random.default_rng(100 + n)
    c, _ = noisy_circuit(n, 40, rng)
    rho = numpy_rho(c, ref.gate_matrix)
    assert abs(np.trace(rho) - 1.0) < 1e-12
    paulis = [(int(rng.integers(0, 1 << n)), int(rng.integers(0, 1 << n))) for _ in range(12)]
    r = ref.run_dm(c, threads=1, paulis=paulis)
    for (x, z), v in zip(paulis, r["terms"]):
        assert abs(v - np.trace(pauli_matrix(n, x, z) @ rho)) < 1e-12
    # The sequence restated through the reference's apply_matrix is rho.
    vec = reference_rho_vector(ref, c)
    dim = 1 << n
    assert np.max(np.abs(vec.reshape(dim, dim).T - rho)) < 1e-12


def test_restatement_known_answers(oracle):
    """The closed forms of the reference's own density-matrix tests
    (tests/engines/density_matrix/density_matrix_engine_test.cpp:132-227)
    on the numpy restatement: no reference build needed."""
    def trace(circ, x, z):
        return np.trace(pauli_matrix(circ.num_qubits, x, z) @ numpy_rho(circ, oracle.gate_matrix))

    def close(a, b):
        return abs(a - b) < 1e-12

    # An empty circuit is |00><00|.
    empty = pyoracle.Circuit(2)
    assert all(close(trace(empty, 0, z), 1.0) for z in range(4))
    assert all(close(trace(empty, x, z), 0.0) for x in range(1, 4) for z in range(4))
    # Depolarizing with p = 0.3: <Z> = 0.7 on |0>, <X> = 0.7 on |+>.
    zero = pyoracle.Circuit(1)
    zero.channel((0,), depolarizing(0.3))
    assert close(trace(zero, 0, 1), 0.7) and close(trace(zero, 1, 0), 0.0) and close(trace(zero, 0, 0), 1.0)
    plus = pyoracle.Circuit(1)
    plus.gate("h", [0])
    plus.channel((0,), depolarizing(0.3))
    assert close(trace(plus, 1, 0), 0.7)
    # Amplitude damping with gamma = 0.25 on |1>: <Z> = 2 gamma - 1.
    one = pyoracle.Circuit(1)
    one.gate("x", [0])
    one.channel((0,), amplitude_damping(0.25))
    assert close(trace(one, 0, 1), -0.5)
    # A one-operator channel whose operator is CX's matrix is the CX gate.
    as_gate = pyoracle.Circuit(2)
    as_gate.gate("h", [0]).gate("ry", [1], [0.4]).gate("cx", [0, 1])
    as_channel = pyoracle.Circuit(2)
    as_channel.gate("h", [0]).gate("ry", [1], [0.4])
    as_channel.channel((0, 1), oracle.gate_matrix(pyoracle.OP["cx"], ())[None])
    # A two-qubit channel K (x) I on operands (1, 0) is K on qubit 1.
    one_q = amplitude_damping(0.4)
    two_q = np.zeros((2, 4, 4), np.complex128)
    for i, k in enumerate(one_q):
        for r in range(4):
            for c in range(4):
                if r >> 1 == c >> 1:
                    two_q[i, r, c] = k[r & 1, c & 1]
    single = pyoracle.Circuit(2)
    single.gate("x", [1]).gate("h", [0])
    single.channel((1,), one_q)
    wide = pyoracle.Circuit(2)
    wide.gate("x", [1]).gate("h", [0])
    wide.channel((1, 0), two_q)
    for x in range(4):
        for z in range(4):
            assert close(trace(as_channel, x, z), trace(as_gate, x, z))
            assert close(trace(wide, x, z), trace(single, x, z))


def test_restated_sequence_is_bitwise_the_reference_engine(ref):
    """The reference engine's traces (trace_with_pauli: a sequential sum,
    density_matrix_engine.cpp:182-197) recomputed on reference_rho_vector
    equal its own to the bit: the restated sequence holds the engine's rho."""
    n = 4
    rng = np.random.default_rng(31)
    c, _ = noisy_circuit(n, 50, rng)
    vec = reference_rho_vector(ref, c)
    paulis = [(int(rng.integers(0, 1 << n)), int(rng.integers(0, 1 << n))) for _ in range(24)]
    r = ref.run_dm(c, threads=1, paulis=paulis)
    powers = [1 + 0j, 1j, -1 + 0j, -1j]
    for (x, z), v in zip(paulis, r["terms"]):
        re = im = 0.0
        for col in range(1 << n):
            e = vec[col | ((col ^ x) << n)]
            if bin(col & z).count("1") % 2:
                re, im = re - e.real, im - e.imag
            else:
                re, im = re + e.real, im + e.imag
        w = powers[bin(x & z).count("1") % 4] * complex(re, im)
        assert (w.real, w.imag) == (v.real, v.imag)


def test_reference_wide_channels_match_numpy(ref):
    n = 5
    rng = np.random.default_rng(77)
    c, _ = noisy_circuit(n, 16, rng, widest=5)
    assert any(len(qs) >= 4 for oc, qs, *_ in c.ops if oc == pyoracle.OP["channel"])
    rho = numpy_rho(c, ref.gate_matrix)
    vec = reference_rho_vector(ref, c)
    dim = 1 << n
    assert np.max(np.abs(vec.reshape(dim, dim).T - rho)) < 1e-12
    paulis = [(int(rng.integers(0, 1 << n)), int(rng.integers(0, 1 << n))) for _ in range(6)]
    r = ref.run_dm(c, threads=1, paulis=paulis)
    for (x, z), v in zip(paulis, r["terms"]):
        assert abs(v - np.trace(pauli_matrix(n, x, z) @ rho)) < 1e-12


def test_reference_dm_counts_follow_the_diagonal(ref):
    n = 4
    rng = np.random.default_rng(7)
    c, _ = noisy_circuit(n, 30, rng)
    rho = numpy_rho(c, ref.gate_matrix)
    t = [(q, q) for q in range(n)]
    shots = 200000
    r = ref.run_dm(c, threads=1, shots=shots, seed=11, targets=t)
    assert sum(r["counts"].values()) == shots
    p = np.real(np.diag(rho))
    for key, cnt in r["counts"].items():
        assert abs(cnt / shots - p[key]) < 5 * np.sqrt(p[key] / shots) + 1e-3


def with_readout_measures(circs, n, rng):
    """Appends measurements of every qubit q into clbit n-1-q to each circuit,
    most with a readout error; clbit n-1 is written twice and the later
    measurement (the one that counts) carries none when n > 1."""
    errs = {}
    for q in range(n):
        if q == 0 and n > 1:
            errs[q] = None
        else:
            e0, e1 = float(rng.uniform(0.02, 0.3)), float(rng.uniform(0.02, 0.3))
            errs[q] = [1.0 - e0, e0, e1, 1.0 - e1]
    for c in circs:
        if n > 1:
            c.measure(0, n - 1, readout=[0.5, 0.5, 0.5, 0.5])  # overwritten below
        for q in range(n):
            c.measure(q, n - 1 - q, readout=errs[q])
    return [(q, n - 1 - q) for q in range(n)]


def restated_readout_counts(ref, circ, shots, seed, targets):
    """The reference's density-matrix counts with readout errors
    (density_matrix_engine.cpp:378-390, src/engines/noise/readout.cpp):
    per shot, one uniform for the true outcome -- the first basis state
    whose sequential cumulative probability exceeds it -- then one per
    readout-errored target, the bit flipping when the uniform is below
    P(recorded != true | true)."""
    import bisect
    n = circ.num_qubits
    vec = reference_rho_vector(ref, circ)
    cum, acc = [], 0.0
    for x in range(1 << n):
        acc += vec[x | (x << n)].real
        cum.append(acc)
    readouts = []
    for _q, cl in targets:
        err = None
        for oc, _qs, _ps, m, c2 in circ.ops:
            if oc == pyoracle.OP["measure"] and c2 == cl:
                err = m
        if err is not None:
            readouts.append((cl, err))
    u = iter(ref.uniforms(seed, shots * (1 + len(readouts))))
    counts = {}
    for _ in range(shots):
        idx = min(bisect.bisect_right(cum, next(u)), len(cum) - 1)
        o = 0
        for q, cl in targets:
            if (idx >> q) & 1:
                o |= 1 << cl
        for cl, a in readouts:
            truth = (o >> cl) & 1
            if next(u) < (a[2] if truth else a[1]):
                o ^= 1 << cl
        counts[o] = counts.get(o, 0) + 1
    return counts


@pytest.mark.parametrize("n", [1, 3])
def test_reference_readout_counts_follow_the_restated_rule(ref, n):
    rng = np.random.default_rng(400 + n)
    c, _ = noisy_circuit(n, 24, rng)
    targets = with_readout_measures([c], n, rng)
    for seed in (3, 4):
        want = ref.run_dm(c, threads=1, shots=3000, seed=seed, targets=targets)["counts"]
        assert restated_readout_counts(ref, c, 3000, seed, targets) == want


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 3, 6])
def test_device_readout_counts_are_the_reference(ctx, ref, n):
    from menos_b200 import DensityMatrix
    rng = np.random.default_rng(500 + n)
    c, d = noisy_circuit(n, 40, rng)
    targets = with_readout_measures([c, d], n, rng)
    rho = DensityMatrix(ctx, n)
    rho.init()
    rho.apply(d)
    for seed in (5, 6):
        got = rho.sample(40000, seed, targets, circuit=d).to_dict()
        assert got == ref.run_dm(c, threads=1, shots=40000, seed=seed, targets=targets)["counts"]
    # Measurements without readout errors: the plain sampler's counts.
    plain = [(q, q) for q in range(n)]
    d2 = type(d)(n)
    d2.ops = [op for op in d.ops if op[0] != pyoracle.OP["measure"]]
    for q in range(n):
        d2.measure(q, q)
    assert rho.sample(5000, 9, plain, circuit=d2).to_dict() == rho.sample(5000, 9, plain).to_dict()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 3, 6, 9])
def test_device_rho_is_bitwise_the_reference(ctx, ref, n):
    from menos_b200 import DensityMatrix
    rng = np.random.default_rng(200 + n)
    c, d = noisy_circuit(n, 60, rng)
    rho = DensityMatrix(ctx, n)
    rho.init()
    rho.apply(d)
    got = rho.state.copy_out()
    want = reference_rho_vector(ref, c)
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
    paulis = [(int(rng.integers(0, 1 << n)), int(rng.integers(0, 1 << n))) for _ in range(16)] + [(0, 0)]
    r = ref.run_dm(c, threads=1, paulis=paulis)
    assert np.max(np.abs(rho.expectation(paulis) - r["terms"])) < 1e-12
    t = [(q, n - 1 - q) for q in range(n)]
    for seed in (1, 2):
        got_counts = rho.sample(50000, seed, t).to_dict()
        assert got_counts == ref.run_dm(c, threads=1, shots=50000, seed=seed, targets=t)["counts"]


@pytest.mark.gpu
@pytest.mark.parametrize("n", [4, 5])
def test_wide_channels_are_bitwise_the_reference(ctx, ref, n):
    """4- and 5-qubit channels: 8- and 10-operand superoperators through the
    wide generic kernel."""
    from menos_b200 import DensityMatrix
    rng = np.random.default_rng(300 + n)
    c, d = noisy_circuit(n, 24, rng, widest=5)
    assert any(len(qs) >= 4 for oc, qs, *_ in d.ops if oc == pyoracle.OP["channel"])
    rho = DensityMatrix(ctx, n)
    rho.init()
    rho.apply(d)
    want = reference_rho_vector(ref, c)
    assert np.array_equal(rho.state.copy_out().view(np.uint64), want.view(np.uint64))
    paulis = [(int(rng.integers(0, 1 << n)), int(rng.integers(0, 1 << n))) for _ in range(8)]
    r = ref.run_dm(c, threads=1, paulis=paulis)
    assert np.max(np.abs(rho.expectation(paulis) - r["terms"])) < 1e-12


@pytest.mark.gpu
def test_dm_of_a_pure_circuit_is_the_outer_product(ctx, oracle):
    from menos_b200 import DensityMatrix, DeviceState
    n = 7
    c = random_circuit(n, 80, np.random.default_rng(3))
    rho = DensityMatrix(ctx, n)
    rho.init()
    rho.apply(c)
    st = DeviceState(ctx, n)
    st.init(c.global_phase)
    st.apply_program(c, fuse_gates=False)
    psi = st.copy_out()
    assert np.max(np.abs(rho.matrix() - np.outer(psi, psi.conj()))) < 1e-13
    paulis = [(int(x), int(z)) for x, z in np.random.default_rng(4).integers(0, 1 << n, size=(10, 2))]
    assert np.max(np.abs(rho.expectation(paulis) - st.expectation(paulis))) < 1e-13


@pytest.mark.gpu
def test_dm_rejects_bad_inputs(ctx):
    from menos_b200 import Circuit, DensityMatrix, DeviceState
    from menos_b200._lib import MB2Error
    rho = DensityMatrix(ctx, 3)
    rho.init()
    with pytest.raises(MB2Error):
        rho.apply(Circuit(3).gate("cx", [0, 5]))
    with pytest.raises(MB2Error):
        rho.expectation([(1 << 3, 0)])
    # A channel on the statevector path is refused with a message.
    st = DeviceState(ctx, 3)
    st.init()
    with pytest.raises(MB2Error, match="density-matrix"):
        st.apply_program(Circuit(3).channel([1], depolarizing(0.1)))
