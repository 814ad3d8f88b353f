"""The fusion plan (mb2_fusion_plan, the plan every sweep applies) against the
known answers of the reference's own fusion tests
(tests/ir/fuse_gates_test.cpp:93-220: ir::plan_fusion's containment rule),
which need no reference build.  Host only."""
import numpy as np
import pytest

from menos_b200._lib import MB2Error
from menos_b200.circuit import Circuit
from menos_b200.engine import fusion_plan


def blocks(c):
    """(member operations, operands) per block, in plan order."""
    order, bb, bq, qb = fusion_plan(c)
    members = [order[bb[b]:bb[b + 1]].tolist() for b in range(len(bb) - 1)]
    operands = [bq[qb[b]:qb[b + 1]].tolist() for b in range(len(qb) - 1)]
    return members, operands


def test_a_gate_joins_the_newest_block_that_contains_or_is_contained():
    # :93-107 -- U(0), U(1), CX(0,1): CX joins U(1)'s block.
    c = Circuit(2).gate("u", [0], [0.1, 0.2, 0.3]).gate("u", [1], [0.4, 0.5, 0.6]).gate("cx", [0, 1])
    assert blocks(c) == ([[0], [1, 2]], [[0], [0, 1]])


def test_a_later_gate_on_a_qubit_of_the_block_joins_it():
    # :109-121
    c = Circuit(3).gate("cx", [0, 1]).gate("u", [0], [0.1, 0.2, 0.3]).gate("u", [1], [0.4, 0.5, 0.6])
    c.gate("h", [2])
    assert blocks(c)[0] == [[0, 1, 2], [3]]


def test_gates_on_different_or_overlapping_qubits_never_merge():
    # :123-134 -- neither set contains the other.
    c = Circuit(5).gate("h", [0]).gate("h", [1]).gate("cx", [2, 3]).gate("cx", [3, 4])
    assert len(blocks(c)[0]) == 4


def test_gates_on_the_same_qubits_merge():
    # :136-147 -- CX(2,1) after CX(1,2): the same set in the other order.
    c = Circuit(3).gate("h", [0]).gate("t", [0]).gate("h", [0]).gate("cx", [1, 2]).gate("cx", [2, 1])
    assert blocks(c) == ([[0, 1, 2], [3, 4]], [[0], [1, 2]])


def test_dense_never_widens_a_diagonal_block_and_vice_versa():
    # :149-168
    c = Circuit(8)
    c.gate("cz", [0, 1]).gate("u", [0], [0.1, 0.2, 0.3])
    c.gate("u", [2], [0.1, 0.2, 0.3]).gate("cz", [2, 3])
    c.gate("rz", [4], [0.7]).gate("cx", [4, 5])
    c.gate("rz", [6], [0.7]).gate("cz", [6, 7]).gate("t", [6])
    assert blocks(c)[0] == [[0], [1], [2], [3], [4, 5], [6, 7, 8]]


def test_a_diagonal_unitary_counts_as_diagonal():
    # :170-195 -- diag(1, i, -1, -i) on {0,1} keeps a dense H(0) apart; the
    # same matrix with one off-diagonal entry takes it.
    diagonal = np.diag([1, 1j, -1, -1j]).astype(np.complex128)
    dense = diagonal.copy()
    dense[0, 1] = 0.5
    assert len(blocks(Circuit(2).unitary([0, 1], diagonal).gate("h", [0]))[0]) == 2
    assert len(blocks(Circuit(2).unitary([0, 1], dense).gate("h", [0]))[0]) == 1


def test_a_measurement_is_a_barrier():
    # :197-207 -- the measurement is a block of its own with no operands.
    c = Circuit(1, 1).gate("h", [0])
    c.measure(0, 0)
    c.gate("h", [0]).gate("t", [0])
    assert blocks(c) == ([[0], [1], [2, 3]], [[0], [], [0]])


def test_an_empty_list_has_no_blocks():
    # :209-214
    order, bb, bq, qb = fusion_plan(Circuit(3))
    assert order.size == 0 and len(bb) - 1 == 0


def test_an_operand_beyond_63_qubits_is_refused():
    # :216-219
    with pytest.raises(MB2Error):
        fusion_plan(Circuit(65).gate("h", [64]))


def test_fusion_plan_size_query():
    """Capacities in, sizes out: a short capacity is refused with the sizes
    set; block_begin and qubits_begin hold one entry more than the blocks."""
    import ctypes as C

    from menos_b200._lib import SweepOptions, lib
    from menos_b200.circuit import to_mb2_ops
    c = Circuit(3).gate("h", [0]).gate("cx", [0, 1]).gate("h", [2])
    arr, keep = to_mb2_ops(c)
    nb, nq = C.c_uint64(0), C.c_uint64(0)
    opts = SweepOptions(1, 0, 0, 0, 0, 0)
    order = np.zeros(3, np.uint32)
    bb = np.zeros(1, np.uint32)
    qb = np.zeros(1, np.uint32)
    bq = np.zeros(1, np.uint32)
    rc = lib().mb2_fusion_plan(arr, 3, C.byref(opts), order.ctypes.data, bb.ctypes.data, bq.ctypes.data,
                               qb.ctypes.data, C.byref(nb), C.byref(nq))
    assert rc != 0 and (nb.value, nq.value) == (2, 3)
    bb = np.zeros(nb.value + 1, np.uint32)
    qb = np.zeros(nb.value + 1, np.uint32)
    bq = np.zeros(nq.value, np.uint32)
    rc = lib().mb2_fusion_plan(arr, 3, C.byref(opts), order.ctypes.data, bb.ctypes.data, bq.ctypes.data,
                               qb.ctypes.data, C.byref(nb), C.byref(nq))
    del keep
    assert rc == 0
    assert (order.tolist(), bb.tolist(), bq.tolist(), qb.tolist()) == ([0, 1, 2], [0, 2, 3], [0, 1, 2], [0, 2, 3])
