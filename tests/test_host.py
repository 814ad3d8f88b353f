"""Host-side product checks that need no GPU: the C ABI's exports, the gate
table, the seeded workloads, and the tiled sweep's block schedule (its
reordering applied on the CPU oracle must be bitwise the plain sweep)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from menos_b200 import _lib, workloads
from menos_b200.circuit import OP, Circuit, to_mb2_ops
from test_oracle_pin import bits_equal, random_circuit


def declared_functions():
    with open(os.path.join(ROOT, "include", "mb2.h")) as f:
        text = f.read()
    return sorted(set(re.findall(r"^int\s+(mb2_\w+)\s*\(", text, flags=re.M)))


def test_every_declared_symbol_is_exported():
    L = C.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(L, name), name
        assert name in _lib.SIGNATURES, name


def test_no_device_is_reported_cleanly():
    # On a machine without a GPU the context refuses loudly; with one it opens.
    h = C.c_void_p()
    rc = _lib.lib().mb2_context_create(0, C.byref(h))
    if rc == 0:
        _lib.lib().mb2_context_destroy(h)
    else:
        assert rc == 4


@pytest.mark.parametrize("opcode", range(21))
def test_gate_table_bitwise(oracle, opcode):
    rng = np.random.default_rng(opcode)
    for _ in range(8):
        p = np.zeros(3)
        p[:] = rng.uniform(-9, 9, size=3)
        out = np.zeros(128, np.float64)
        assert _lib.lib().mb2_gate_matrix(opcode, p.ctypes.data, out.ctypes.data, 128) == 0
        ref = oracle.gate_matrix(opcode, p)
        assert bits_equal(out[:2 * ref.size], ref.view(np.float64).ravel())


def gate(name, params=()):
    p = np.zeros(3)
    p[:len(params)] = params
    out = np.zeros(128, np.float64)
    assert _lib.lib().mb2_gate_matrix(OP[name], p.ctypes.data, out.ctypes.data, 128) == 0
    k = 3 if name == "ccx" else (2 if name in ("cx", "cz", "swap", "cp", "rzz") else 1)
    d = 1 << k
    return out[:2 * d * d].view(np.complex128).reshape(d, d)


def test_gate_table_known_answers():
    # tests/ir/gate_table_test.cpp:105-190.  RZZ(t) is diagonal with
    # e^{-it/2} on |00>, |11> and e^{it/2} on |01>, |10>, and equals
    # CX RZ(t) CX (RZ on operand 1, CX flipping bit 1 when bit 0 is set).
    t = 0.83
    rzz = gate("rzz", [t])
    want = np.diag([np.exp(-0.5j * t), np.exp(0.5j * t), np.exp(0.5j * t), np.exp(-0.5j * t)])
    assert np.max(np.abs(rzz - want)) <= 1e-15
    rz = gate("rz", [t])
    for i in range(4):
        flipped = i ^ 2 if i & 1 else i
        assert abs(rzz[i, i] - rz[(flipped >> 1) & 1, (flipped >> 1) & 1]) <= 1e-15
    # RZ is not P: they differ by a global phase.
    assert abs(gate("rz", [1.234])[0, 0] - gate("p", [1.234])[0, 0]) > 1e-6
    # CX operands are (control, target) = (bit 0, bit 1): |control set> at
    # local index 1 goes to index 3.
    cx = gate("cx")
    assert cx[3, 1] == 1.0 and cx[1, 1] == 0.0


def test_gate_table_rejects_non_gates():
    out = np.zeros(128, np.float64)
    assert _lib.lib().mb2_gate_matrix(OP["unitary"], None, out.ctypes.data, 128) == 1
    assert _lib.lib().mb2_gate_matrix(OP["measure"], None, out.ctypes.data, 128) == 1


def test_workload_rng_is_mt19937_64(oracle):
    for seed in (0, 5, 20260929):
        rng = workloads.MT19937_64(seed)
        ours = [rng.next_word() for _ in range(700)]
        assert ours == [int(w) for w in oracle.words(seed, 700)]


def test_workload_shapes():
    c1 = workloads.config_c1()
    assert sum(1 for o in c1.ops if o[0] == OP["u"]) == 400
    assert sum(1 for o in c1.ops if o[0] == OP["cz"]) == 190
    c2 = workloads.config_c2()
    assert sum(1 for o in c2.ops if o[0] == OP["u"]) == 1200
    assert sum(1 for o in c2.ops if o[0] == OP["cz"]) == 580
    assert sum(1 for o in c2.ops if o[0] == OP["cp"]) == 435
    assert sum(1 for o in c2.ops if o[0] == OP["swap"]) == 15
    h = workloads.hea(16, 8, 1)
    assert sum(1 for o in h.ops if o[0] == OP["cx"]) == 8 * 15
    ps = workloads.pauli_strings(30, 64, 3)
    assert len(ps) == 64 and all(x < (1 << 30) and z < (1 << 30) for x, z in ps)


def schedule(circ, n, fuse=True, tile=0, per_gate=False, precision=_lib.C128):
    arr, keep = to_mb2_ops(circ)
    opts = _lib.SweepOptions(1 if fuse else 0, 0, tile, 1 if per_gate else 0)
    cap = 4 * len(circ.ops) + 4
    pas = np.zeros(cap, np.uint32)
    ks = np.zeros(cap, np.uint32)
    qs = np.zeros(6 * cap, np.uint32)
    mats = np.zeros(cap * 2 * 4096, np.float64)
    nb = C.c_uint64(cap)
    ml = C.c_uint64(mats.size)
    rc = _lib.lib().mb2_debug_schedule(arr, len(circ.ops), C.byref(opts), n, pas.ctypes.data, ks.ctypes.data,
                                       qs.ctypes.data, mats.ctypes.data, C.byref(nb), C.byref(ml), precision)
    assert rc == 0
    out, off = [], 0
    for i in range(nb.value):
        k = int(ks[i])
        d = 1 << k
        m = mats[off:off + 2 * d * d].view(np.complex128).reshape(d, d)
        off += 2 * d * d
        out.append((int(pas[i]), list(qs[6 * i:6 * i + k]), m))
    return out


def as_oracle_circuit(c):
    import pyoracle
    oc = pyoracle.Circuit(c.num_qubits, c.global_phase)
    oc.ops = list(c.ops)
    return oc


@pytest.mark.parametrize("tile", [4, 5, 7, 12])
def test_tiled_schedule_is_bitwise_the_plain_sweep(oracle, tile):
    rng = np.random.default_rng(tile)
    for n in (4, 6, 9, 11, 13):
        for fuse in (True, False):
            c = random_circuit(n, 80, rng)
            c.num_clbits = 0
            sched = schedule(c, n, fuse=fuse, tile=tile)
            state = oracle.initialize(n, c.global_phase)
            passes = [p for p, _, _ in sched]
            assert passes == sorted(passes)
            for _p, qs, m in sched:
                oracle.apply_generic(state, m, qs)
            expect = oracle.run(as_oracle_circuit(c), fuse_gates=fuse)
            assert bits_equal(state, expect), (n, fuse, tile)


@pytest.mark.parametrize("tile", [4, 5, 7, 12, 13])
def test_complex64_schedule_is_a_dependency_order(oracle, tile):
    # The complex64 planner reorders blocks on disjoint qubits: every qubit
    # sees its blocks in plan order, and the state is the in-order one up to
    # rounding.
    rng = np.random.default_rng(100 + tile)
    for n in (4, 6, 9, 13, 16):
        for fuse in (True, False):
            c = random_circuit(n, 80, rng)
            c.num_clbits = 0
            plain = schedule(c, n, fuse=fuse, tile=tile)
            reord = schedule(c, n, fuse=fuse, tile=tile, precision=_lib.C64)
            assert len(plain) == len(reord)
            passes = [p for p, _, _ in reord]
            assert passes == sorted(passes)
            key = lambda qs, m: (tuple(int(q) for q in qs), m.tobytes())
            for q in range(n):
                seq_p = [key(qs, m) for _, qs, m in plain if q in qs]
                seq_r = [key(qs, m) for _, qs, m in reord if q in qs]
                assert seq_p == seq_r, (n, fuse, tile, q)
            state = oracle.initialize(n, c.global_phase)
            for _p, qs, m in reord:
                oracle.apply_generic(state, m, qs)
            expect = oracle.run(as_oracle_circuit(c), fuse_gates=fuse)
            assert np.max(np.abs(state - expect)) < 1e-12, (n, fuse, tile)


def test_complex64_brick_schedule_has_few_passes():
    # Light-cone tiles: a 12-qubit tile runs several brick layers of its
    # qubits before the next tile, instead of one run of consecutive blocks.
    c = workloads.brick(28, 32, 5)
    plain = max(p for p, _, _ in schedule(c, 28, tile=12)) + 1
    reord = max(p for p, _, _ in schedule(c, 28, tile=12, precision=_lib.C64)) + 1
    assert reord <= 40 and 3 * reord <= plain, (reord, plain)


def test_brick_schedule_pass_count():
    c = workloads.brick(30, 40, 1)
    workloads.qft(30, c)
    sched = schedule(c, 30, fuse=True, tile=12)
    passes = max(p for p, _, _ in sched) + 1
    # runs of consecutive blocks (never reordered), diagonals reading qubits
    # outside the tile: ~160 passes instead of one per block (2260 blocks)
    assert passes < 200, passes


def test_packed_circuit_is_the_same_op_array():
    from menos_b200.circuit import PackedCircuit, to_mb2_ops
    c = workloads.config_c2(n=10, depth=3)
    c.unitary([1, 4], np.eye(4, dtype=np.complex128))
    c.measure(2, 0)
    p = PackedCircuit(c)
    a, _ = to_mb2_ops(c)
    b, _ = to_mb2_ops(p)
    assert len(p) == len(c.ops) and p.num_qubits == c.num_qubits and p.global_phase == c.global_phase
    assert p.measure_targets() == c.measure_targets()
    for x, y in zip(a[:len(c.ops)], b[:len(c.ops)]):
        assert (x.opcode, x.num_qubits, list(x.qubits), list(x.params), x.clbit) == \
               (y.opcode, y.num_qubits, list(y.qubits), list(y.params), y.clbit)
        assert bool(x.matrix) == bool(y.matrix)
    assert to_mb2_ops(p)[0] is b  # packed once, reused
