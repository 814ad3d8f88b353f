"""The complex128 plan with diagonal operands outside the tile, on the CPU.

A pass applies a run of consecutive blocks; a diagonal block may read up to
16 qubits outside the pass's tile (one bit value per tile).  Through
mb2_debug_run_plan the planned program -- every block in plan order, each
diagonal's operands mapped to tile positions or to the outside qubits --
interpreted on the host gives the oracle's state, and the headline circuit
needs far fewer passes than with every operand inside the tile.
"""
import ctypes as C

import numpy as np
import pytest

from menos_b200 import _lib, workloads
from menos_b200.circuit import Circuit, to_mb2_ops
from test_host import as_oracle_circuit, schedule
from test_oracle_pin import random_circuit

C128 = _lib.C128


def run_plan(circ, tile=0, fuse=True):
    arr, keep = to_mb2_ops(circ)
    n = circ.num_qubits
    st = np.zeros(1 << n, np.complex128)
    st[0] = np.exp(1j * circ.global_phase)
    stats = np.zeros(6, np.uint64)
    opts = _lib.SweepOptions(1 if fuse else 0, 0, tile, 0, 0)
    rc = _lib.lib().mb2_debug_run_plan(arr, len(circ.ops), C.byref(opts), n, C128, st.ctypes.data,
                                       stats.ctypes.data)
    assert rc == 0
    del keep
    return st, int(stats[0])


def diagonal_heavy(n, layers, seed):
    """CZ / CP / RZZ / CCZ-like diagonals on far-apart qubits between U3 layers."""
    rng = np.random.default_rng(seed)
    c = Circuit(n)
    for _ in range(layers):
        for q in range(n):
            c.gate("u", [q], rng.uniform(-3, 3, 3))
        for _ in range(n):
            a, b = (int(v) for v in rng.choice(n, 2, replace=False))
            kind = rng.integers(0, 4)
            if kind == 0:
                c.gate("cz", [a, b])
            elif kind == 1:
                c.gate("cp", [a, b], [rng.uniform(-3, 3)])
            elif kind == 2:
                c.gate("rzz", [a, b], [rng.uniform(-3, 3)])
            else:
                qs = [int(v) for v in rng.choice(n, 3, replace=False)]
                c.unitary(qs, np.diag([1, 1, 1, 1, 1, 1, 1, -1]).astype(np.complex128))
        c.gate("rz", [int(rng.integers(0, n))], [rng.uniform(-3, 3)])
    return c


@pytest.mark.parametrize("tile", [4, 6, 9, 11, 12])
def test_plans_with_outside_operands_give_the_oracle_state(oracle, tile):
    n = 14
    for seed in range(3):
        for c in (diagonal_heavy(n, 4, seed), random_circuit(n, 150, np.random.default_rng(seed))):
            for fuse in (True, False):
                got, _ = run_plan(c, tile=tile, fuse=fuse)
                want = oracle.run(as_oracle_circuit(c), fuse_gates=fuse)
                assert np.max(np.abs(got - want)) < 1e-12, (tile, seed, fuse)


def test_headline_circuit_needs_fewer_passes():
    # Brick depth 40 + QFT: a brick layer's CZs and the QFT's controlled
    # phases no longer end a pass when their qubits leave the tile.
    for n, most in ((28, 170), (30, 185)):
        c = workloads.config_c2(n=n, depth=40)
        passes = max(p for p, _, _ in schedule(c, n)) + 1
        assert passes <= most, (n, passes)


def test_block_order_is_unchanged():
    # Only the pass boundaries move: the application order is the plan order.
    c = workloads.config_c2(n=20, depth=6)
    s = schedule(c, 20)
    plain = schedule(c, 20, per_gate=True)
    assert [q for _, q, _ in s] == [q for _, q, _ in plain]
