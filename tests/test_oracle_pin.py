"""Pins the CPU oracle (oracle/oracle.c) to the reference: against the
reference's own CPU engine compiled here (oracle/_ref) and against the
reference's golden values (tests/golden/, made by tests/golden/make_golden.py).
CPU only."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from pyoracle import OP, Circuit

RNG = np.random.default_rng(20260929)


def rand_state(n, rng=RNG):
    s = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return (s / np.linalg.norm(s)).astype(np.complex128)


def rand_unitary(k, rng=RNG):
    a = rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))
    q, r = np.linalg.qr(a)
    return (q * (np.diag(r) / np.abs(np.diag(r)))).astype(np.complex128)


def bits_equal(a, b):
    return np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))


def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


# --- golden vectors (no reference library needed) ---------------------------

def test_golden_counts_seed42_plus_state(oracle):
    # tests/engines/dense/sample_test.cpp:85-97: 20 shots of |+> at seed 42.
    plus = np.array([1, 1], np.complex128) / np.sqrt(2.0)
    assert oracle.sample(plus, 20, 42, [(0, 0)]) == {0: 9, 1: 11}


def test_sampler_known_answers(oracle):
    # tests/engines/dense/sample_test.cpp:39-83: zero shots give no counts;
    # the same seed gives the same counts; every shot is counted; basis bits
    # reach clbits through the targets (|q1=1, q0=0>, q0 -> c1, q1 -> c0:
    # outcome 1).
    plus = np.array([1, 1], np.complex128) / np.sqrt(2.0)
    assert oracle.sample(plus, 0, 1, [(0, 0)]) == {}
    assert oracle.sample(plus, 1000, 2024, [(0, 0)]) == oracle.sample(plus, 1000, 2024, [(0, 0)])
    assert sum(oracle.sample(plus, 12345, 9, [(0, 0)]).values()) == 12345
    basis2 = np.array([0, 0, 1, 0], np.complex128)
    assert oracle.sample(basis2, 10, 1, [(0, 1), (1, 0)]) == {1: 10}


def test_sampler_chi_square(oracle):
    # tests/engines/dense/sample_test.cpp:99-127: 1e5 shots of probabilities
    # 0.1..0.4 at seed 31415 stay below the chi-square critical value for
    # three degrees of freedom at 0.001 (16.2662).
    p = np.array([0.1, 0.2, 0.3, 0.4])
    counts = oracle.sample(np.sqrt(p).astype(np.complex128), 100000, 31415, [(0, 0), (1, 1)])
    obs = np.array([counts.get(k, 0) for k in range(4)], float)
    assert float(np.sum((obs - p * 1e5) ** 2 / (p * 1e5))) < 16.2662


# tests/engines/dense/dense_engine_test.cpp:279-330, Y = i X Z (Qiskit's
# convention): (qubits, gates, [(x mask, z mask, <P>)]) for S H|0>,
# S(0) CX(0,1) H(0)|00> and the product (S H|0>)(H|0>)(S H|0>).
Y_CONVENTION = [
    (1, [("h", [0]), ("s", [0])], [(1, 1, 1.0), (1, 0, 0.0), (0, 1, 0.0)]),
    (2, [("h", [0]), ("cx", [0, 1]), ("s", [0])],
     [(0b11, 0b10, 1.0), (0b11, 0b01, 1.0), (0b00, 0b11, 1.0), (0b11, 0b11, 0.0), (0b11, 0b00, 0.0)]),
    (3, [("h", [0]), ("s", [0]), ("h", [1]), ("h", [2]), ("s", [2])],
     [(0b001, 0b001, 1.0), (0b010, 0b010, 0.0), (0b100, 0b100, 1.0), (0b101, 0b101, 1.0),
      (0b011, 0b011, 0.0), (0b001, 0b000, 0.0), (0b000, 0b001, 0.0)]),
]


def test_y_convention_known_answers(oracle):
    for n, gates, terms in Y_CONVENTION:
        c = Circuit(n)
        for name, qs in gates:
            c.gate(name, qs)
        s = oracle.run(c)
        for x, z, want in terms:
            assert abs(oracle.expectation(s, x, z) - want) <= 1e-12, (n, x, z)


def test_golden_fixtures(oracle):
    g = golden()
    for case in g["uniforms"]:
        u = oracle.uniforms(case["seed"], len(case["hex"]))
        assert [v.hex() for v in u] == case["hex"]
    for case in g["gate_matrices"]:
        m = oracle.gate_matrix(case["opcode"], case["params"])
        assert [float.hex(float(x)) for x in m.view(np.float64).ravel()] == case["hex"], case
    for case in g["circuits"]:
        c = Circuit(case["n"], case["global_phase"])
        for oc, qs, ps in case["ops"]:
            c.gate(oc, qs, ps)
        sv = oracle.run(c, fuse_gates=case["fuse"])
        assert [float.hex(float(x)) for x in sv.view(np.float64)] == case["statevector_hex"], case["name"]
        counts = oracle.sample(sv, case["shots"], case["seed"], [(q, q) for q in range(case["n"])])
        assert {str(k): v for k, v in counts.items()} == case["counts"], case["name"]
        for (x, z), (re, im) in zip(case["paulis"], case["terms"]):
            v = oracle.expectation(sv, x, z)
            assert v.real.hex() == re and v.imag.hex() == im


# --- against the reference library --------------------------------------------

@pytest.mark.parametrize("opcode", range(21))
def test_gate_matrices_bitwise(oracle, ref, opcode):
    for _ in range(6):
        params = list(RNG.uniform(-7, 7, size=3))
        assert bits_equal(oracle.gate_matrix(opcode, params), ref.gate_matrix(opcode, params))


def test_generic_kernel_bitwise_every_operand_order(oracle, ref):
    n = 7
    for k in range(1, 6):
        for trial in range(6):
            ops = RNG.permutation(n)[:k]
            u = rand_unitary(k)
            s0 = rand_state(n)
            a, b, c = s0.copy(), s0.copy(), s0.copy()
            oracle.apply_generic(a, u, ops)
            ref.apply_matrix(b, u, ops, threads=1)
            ref.apply_matrix(c, u, ops, threads=1, generic=True)
            assert bits_equal(a, b) and bits_equal(a, c), (k, ops)


def test_dispatch_paths_bitwise(oracle, ref):
    # diagonal / 1q / 2q specialisations of the reference equal its generic kernel
    n = 18  # above kParallelMinGroups so the threaded sweep runs
    s0 = rand_state(n)
    for name, qs, ps in [("rz", [5], [0.3]), ("u", [0], [0.1, 0.2, 0.3]), ("u", [13], [1.1, 2.2, 3.3]),
                         ("cx", [3, 1], []), ("cp", [17, 2], [0.7]), ("ccx", [4, 0, 9], [])]:
        m = oracle.gate_matrix(OP[name], ps)
        a, b = s0.copy(), s0.copy()
        oracle.apply_generic(a, m, qs)
        ref.apply_matrix(b, m, qs, threads=ref.default_threads())
        assert bits_equal(a, b), name


def test_expectation_bitwise(oracle, ref):
    n = 9
    s = rand_state(n)
    for _ in range(20):
        x, z = int(RNG.integers(0, 1 << n)), int(RNG.integers(0, 1 << n))
        assert oracle.expectation(s, x, z) == ref.expectation(s, x, z)


def test_uniforms_and_sampling(oracle, ref):
    for seed in [0, 1, 42, 2 ** 63 + 5]:
        assert bits_equal(oracle.uniforms(seed, 1000), ref.uniforms(seed, 1000))
    s = rand_state(10)
    for shots, seed in [(1, 3), (4096, 7), (20000, 99)]:
        t = [(q, q) for q in range(10)]
        assert oracle.sample(s, shots, seed, t) == ref.sample(s, shots, seed, t)
    # measure-target remapping and partial measurement
    t = [(3, 0), (7, 1), (0, 5)]
    assert oracle.sample(s, 5000, 11, t) == ref.sample(s, 5000, 11, t, width=6)


def random_circuit(n, n_ops, rng, unitaries=True):
    c = Circuit(n, float(rng.uniform(-3, 3)))
    names = ["x", "y", "z", "h", "s", "sdg", "t", "tdg", "sx", "sxdg", "rx", "ry", "rz", "p", "u", "cx", "cz",
             "swap", "cp", "rzz", "ccx"]
    for _ in range(n_ops):
        r = rng.random()
        if unitaries and r < 0.1:
            k = int(rng.integers(1, min(5, n) + 1))
            c.unitary(rng.permutation(n)[:k], rand_unitary(k, rng))
            continue
        name = names[int(rng.integers(0, len(names)))]
        nq = 1 if OP[name] <= 14 else (3 if name == "ccx" else 2)
        if nq > n:
            continue
        qs = rng.permutation(n)[:nq]
        npar = {"rx": 1, "ry": 1, "rz": 1, "p": 1, "cp": 1, "rzz": 1, "u": 3}.get(name, 0)
        c.gate(name, qs, rng.uniform(-7, 7, size=npar))
    return c


def test_plan_fusion_equal(oracle, ref):
    rng = np.random.default_rng(987654321)
    for trial in range(20):
        c = random_circuit(8, 60, rng)
        a = oracle.plan_fusion(c)
        b = ref.plan_fusion(c)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
        blocks = len(a[1]) - 1
        for blk in range(blocks):
            if a[1][blk + 1] - a[1][blk] >= 2:
                assert bits_equal(oracle.fused_block_matrix(c, blk), ref.fused_block_matrix(c, blk))


def test_run_bitwise_random_circuits(oracle, ref):
    rng = np.random.default_rng(987654321)
    for n in range(1, 11):
        for fuse in (False, True):
            c = random_circuit(n, 40, rng)
            a = oracle.run(c, fuse_gates=fuse)
            b = ref.run(c, fuse_gates=fuse, threads=1)["statevector"]
            assert bits_equal(a, b), (n, fuse)
