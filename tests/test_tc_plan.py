"""The complex64 plans on the CPU, through mb2_debug_run_plan: the commuting
pass order and its tensor-core form (each phase's dense gates composed into
one 16x16 matrix, diagonals on thread qubits applied before or after it,
passes split when their matrices overflow shared memory), interpreted in FP64
on the host, give the oracle's state within 1e-12 -- so any error of the
device path beyond that is the kernel's arithmetic, not the plan's."""
import ctypes as C

import numpy as np
import pytest

from menos_b200 import _lib, workloads
from menos_b200.circuit import Circuit, to_mb2_ops
from menos_b200.engine import C64
from test_host import as_oracle_circuit


def run_plan(circ, tile=0, kernel=2, fuse=True):
    arr, keep = to_mb2_ops(circ)
    n = circ.num_qubits
    st = np.zeros(1 << n, np.complex128)
    st[0] = 1.0
    stats = np.zeros(6, np.uint64)
    opts = _lib.SweepOptions(1 if fuse else 0, 0, tile, 0, kernel)
    rc = _lib.lib().mb2_debug_run_plan(arr, len(circ.ops), C.byref(opts), n, C64, st.ctypes.data, stats.ctypes.data)
    assert rc == 0
    del keep
    return st, {"passes": int(stats[0]), "tc_passes": int(stats[1]), "matrices": int(stats[2]), "tile": int(stats[3])}


def mixed_circuit(n, layers, seed):
    """Every gate kind the engine takes, on random operands."""
    rng = np.random.default_rng(seed)
    c = Circuit(n)
    one = ["x", "y", "z", "h", "s", "sdg", "t", "tdg", "sx", "sxdg"]
    for _ in range(layers):
        for q in range(n):
            k = rng.integers(0, 5)
            if k == 0:
                c.gate(one[rng.integers(0, len(one))], [q])
            elif k == 1:
                c.gate("u", [q], rng.uniform(0, 2 * np.pi, 3))
            else:
                c.gate(["rx", "ry", "rz", "p"][rng.integers(0, 4)], [q], [rng.uniform(-4, 4)])
        for _ in range(n // 2):
            a, b = rng.permutation(n)[:2]
            name = ["cx", "cz", "swap", "cp", "rzz"][rng.integers(0, 5)]
            c.gate(name, [a, b], [rng.uniform(-4, 4)] if name in ("cp", "rzz") else [])
        if rng.integers(0, 3) == 0:
            c.gate("ccx", list(rng.permutation(n)[:3]))
    return c


CIRCUITS = {
    "brick": lambda n: workloads.brick(n, 10, 3),
    "brick+qft": lambda n: workloads.qft(n, workloads.brick(n, 4, 5)),
    "hea": lambda n: workloads.hea(n, 6, 7),
    "mixed": lambda n: mixed_circuit(n, 6, n),
}


@pytest.mark.parametrize("name", sorted(CIRCUITS))
@pytest.mark.parametrize("n,tile", [(14, 12), (15, 13), (16, 12)])
def test_tensor_core_plan_matches_oracle(oracle, name, n, tile):
    circ = CIRCUITS[name](n)
    expect = oracle.run(as_oracle_circuit(circ), fuse_gates=True)
    got, stats = run_plan(circ, tile=tile)
    assert stats["tile"] == tile
    if name != "mixed":  # a pass with a three-qubit block stays on the SIMT kernel
        assert stats["tc_passes"] > 0 and stats["matrices"] > 0
    assert np.max(np.abs(got - expect)) <= 1e-12
    # The FP32 SIMT form of the same plan, for comparison.
    simt, s2 = run_plan(circ, tile=tile, kernel=1)
    assert s2["tc_passes"] == 0
    assert np.max(np.abs(simt - expect)) <= 1e-12


def test_split_passes_keep_the_order(oracle):
    # Deep circuits on few qubits: one tile holds the whole state, so a pass
    # carries many phases and is split at the shared-memory limit.
    circ = workloads.brick(12, 40, 9)
    got, stats = run_plan(circ, tile=12)
    _, simt = run_plan(circ, tile=12, kernel=1)
    assert stats["tc_passes"] == stats["passes"] > simt["passes"]
    expect = oracle.run(as_oracle_circuit(circ), fuse_gates=True)
    assert np.max(np.abs(got - expect)) <= 1e-12
