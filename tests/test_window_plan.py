"""The window plan of the chunked tier on the copy engines
(mb2_window_plan, what mb2_apply_program_windowed runs) against the
reference's own pass planner compiled from its sources
(src/engines/dense_tiered/pass_plan.cpp: build_pass_plan's greedy rule over
the fusion plan's blocks, choose_pass_plan's chunk choice), and against the
known answers of the reference's own pass-plan tests, which need no
reference build."""
import ctypes as C

import numpy as np
import pytest

import pyoracle
from menos_b200 import workloads
from menos_b200._lib import SweepOptions, lib
from menos_b200.circuit import Circuit, to_mb2_ops
from test_oracle_pin import random_circuit


def window_plan(circ, window, chunk, fuse=1):
    """(L, [(global mask, first block, end block), ...]), or None when refused."""
    arr, keep = to_mb2_ops(circ)
    out = (C.c_uint64 * (1 << 18))()
    nw = C.c_uint64(1 << 18)
    opts = SweepOptions(fuse, 0, 0, 0, 0, 0)
    rc = lib().mb2_window_plan(arr, len(circ.ops), C.byref(opts), circ.num_qubits, window, chunk, out, C.byref(nw))
    del keep
    if rc != 0:
        return None
    w = list(out[:nw.value])
    return w[0], [tuple(w[3 + 3 * i:6 + 3 * i]) for i in range(w[2])]


def as_oracle(c):
    o = pyoracle.Circuit(c.num_qubits, c.global_phase)
    o.ops = list(c.ops)
    return o


CIRCUITS = [("c2", lambda n: workloads.config_c2(n=n, depth=10)), ("hea", lambda n: workloads.hea(n, 6, 3)),
            ("random", lambda n: random_circuit(n, 180, np.random.default_rng(n)))]


@pytest.mark.parametrize("name,make", CIRCUITS)
@pytest.mark.parametrize("n,window,chunk", [(16, 12, 8), (16, 14, 10), (18, 15, 5), (20, 20, 12)])
def test_greedy_passes_are_the_reference(ref, name, make, n, window, chunk):
    c = make(n)
    L, too_small, passes = ref.pass_plan(as_oracle(c), chunk, window)
    mine = window_plan(c, window, chunk)
    if too_small:
        assert mine is None
    else:
        assert mine == (L, passes)


@pytest.mark.parametrize("name,make", CIRCUITS)
@pytest.mark.parametrize("n,window", [(30, 27), (34, 31), (32, 26)])
def test_chunk_choice_is_the_reference(ref, name, make, n, window):
    """Windows above 2^24 amplitudes: the chunk with the fewest passes, the
    larger on a tie, as choose_pass_plan picks it."""
    c = make(n)
    L, _too_small, passes = ref.pass_plan(as_oracle(c), 0, window)
    assert window_plan(c, window, 0) == (L, passes)


def test_small_windows_keep_chunks_of_at_least_2_16(ref):
    """Windows of at most 2^24 amplitudes: the same rule (fewest passes,
    larger chunk on a tie) searched from the window down to 2^min(16, W)
    only (the reference goes on down to one amplitude), smaller chunks only
    when none of those fits."""
    n = 22
    c = workloads.config_c2(n=n, depth=6)
    for window in (18, 20):
        L, passes = window_plan(c, window, 0)
        assert 16 <= L <= window
        best = min((len(window_plan(c, window, l)[1]), -l) for l in range(16, window + 1)
                   if window_plan(c, window, l) is not None)
        assert (len(passes), -L) == best
    # A window too narrow for chunks of 2^16 still finds a plan below it.
    L, passes = window_plan(c, 12, 0)
    assert L < 12 and passes


# ---- the reference's own known answers (tests/engines/dense_tiered/
# pass_plan_test.cpp), on the unfused operation list as there: one block per
# gate, MeasureOps are no block here (the reference counts them inside a
# pass's operation range).  Its small cases use chunks of 2^2 and 2^3
# amplitudes, below the tile kernels' 2^4: they are restated one or two
# qubits higher (every qubit index shifted up), which leaves every global
# mask and pass boundary as it was.

@pytest.mark.parametrize("make,n,chunk,window,passes", [
    # StepOnePassCountsOfTheCrossoverFamilyArePinned (:156-172)
    (workloads.crossover, 31, 27, 29, 24), (workloads.crossover, 31, 27, 30, 13),
    (workloads.crossover, 31, 27, 31, 1), (workloads.crossover, 31, 28, 30, 15),
    (workloads.crossover, 31, 25, 27, 36), (workloads.crossover, 31, 25, 29, 18),
    (workloads.crossover, 31, 24, 28, 21), (workloads.crossover, 33, 28, 30, 30),
    (workloads.crossover, 33, 27, 29, 36), (workloads.crossover, 33, 24, 28, 27),
    # StepOnePassCountsOfTheLadderFamilyArePinned (:174-181)
    (workloads.ladder, 31, 27, 29, 30), (workloads.ladder, 31, 28, 30, 24),
    (workloads.ladder, 31, 24, 28, 24), (workloads.ladder, 31, 24, 26, 60)])
def test_reference_pinned_pass_counts(make, n, chunk, window, passes):
    c = make(n)
    if n == 31:  # the families' sizes the reference pins beside the counts
        assert len(c.ops) == (282 if make is workloads.crossover else 366)
    L, got = window_plan(c, window, chunk, fuse=0)
    assert (L, len(got)) == (chunk, passes)


def test_reference_pinned_global_operands():
    # build_pass_plan(crossover(31), 31, 27, 29): 36 gates touch a global
    # qubit, at most two global operands each (:166-167).
    c = workloads.crossover(31)
    L, passes = window_plan(c, 29, 27, fuse=0)
    touching = sum(1 for _, qs, *_ in c.ops if any(q >= L for q in qs))
    assert touching == 36
    assert max(sum(1 for q in qs if q >= L) for _, qs, *_ in c.ops) == 2
    assert all(bin(mask).count("1") <= 29 - 27 for mask, _, _ in passes)


def test_reference_pinned_chunk_choice():
    # ChoosesTheChunkSizeWithTheFewestPassesLargerOnATie (:183-197): in a
    # 2^29 window the crossover circuit at 31 qubits takes chunks of 2^25
    # (18 passes against 24 with 2^27); a window holding the whole state is
    # one pass at the largest chunk.
    L, passes = window_plan(workloads.crossover(31), 29, 0, fuse=0)
    assert (L, len(passes)) == (25, 18)
    L, passes = window_plan(workloads.crossover(12), 12, 0, fuse=0)
    assert (L, len(passes)) == (12, 1)


def test_reference_no_gate_no_pass():
    # ACircuitWithNoGateHasNoPass (:54-61), at a 2^4 chunk.
    c = Circuit(6, 6)
    c.measure(0, 0)
    assert window_plan(c, 5, 4, fuse=0) == (4, [])


def test_reference_local_gates_one_pass_with_an_empty_group():
    # LocalGatesOnlyAreOnePassWithAnEmptyGroup (:63-76), one qubit higher.
    c = Circuit(7)
    for q in range(3):
        c.gate("h", [q + 1])
    c.gate("cx", [1, 3])
    assert window_plan(c, 4, 4, fuse=0) == (4, [(0, 0, 4)])


def test_reference_greedy_rule_extends_and_closes():
    # TheGreedyRuleExtendsAGroupWhileItFitsAndClosesOtherwise (:78-104), one
    # qubit higher: chunk 2^4, globals 4, 5, 6 (mask bits 0, 1, 2).
    c = Circuit(7, 6)
    c.gate("cx", [1, 4])   # G = {4}
    c.gate("h", [2])       # local, same pass
    c.gate("cx", [5, 2])   # G = {4, 5}: fits two
    c.measure(1, 0)        # same pass
    c.gate("cx", [6, 1])   # {4, 5, 6} does not fit: new pass, G = {6}
    c.gate("cx", [4, 6])   # G = {4, 6}
    c.measure(2, 1)
    assert window_plan(c, 6, 4, fuse=0) == (4, [(0b011, 0, 3), (0b101, 3, 5)])
    assert window_plan(c, 7, 4, fuse=0) == (4, [(0b111, 0, 5)])


def test_reference_one_pass_per_gate_when_the_window_holds_one():
    # EveryGateGlobalGivesOnePassPerGateWhenTheWindowHoldsOne (:106-117),
    # two qubits higher.
    c = Circuit(6)
    for q in (4, 5, 4):
        c.gate("h", [q])
    assert window_plan(c, 5, 4, fuse=0) == (4, [(0b01, 0, 1), (0b10, 1, 2), (0b01, 2, 3)])


def test_reference_too_many_global_operands_is_refused():
    # AGateWithMoreGlobalOperandsThanTheWindowHoldsIsReported (:119-131), one
    # qubit higher: a 5-qubit unitary on five global qubits.
    c = Circuit(9)
    c.unitary([4, 5, 6, 7, 8], np.eye(32))
    assert window_plan(c, 8, 4, fuse=0) is None
    assert window_plan(c, 9, 4, fuse=0) == (4, [(0b11111, 0, 1)])


def test_reference_passes_partition_the_blocks_in_order():
    # PassesPartitionTheOperationsInOrder (:133-150).
    c = workloads.crossover(12)
    for chunk in range(6, 13):
        for window in range(chunk, 13):
            r = window_plan(c, window, chunk, fuse=0)
            if r is None:
                continue
            passes = r[1]
            assert passes and passes[0][1] == 0 and passes[-1][2] == len(c.ops)
            for a, b in zip(passes, passes[1:]):
                assert b[1] == a[2] and b[1] < b[2]


def test_argument_refusals_and_capacity():
    c = workloads.crossover(12)
    arr, keep = to_mb2_ops(c)
    opts = SweepOptions(0, 0, 0, 0, 0, 0)
    out = (C.c_uint64 * 64)()

    def call(n, window, chunk, cap):
        nw = C.c_uint64(cap)
        rc = lib().mb2_window_plan(arr, len(c.ops), C.byref(opts), n, window, chunk, out, C.byref(nw))
        return rc, nw.value

    assert call(12, 3, 0, 64)[0] != 0          # a window below 2^4 amplitudes
    assert call(12, 13, 0, 64)[0] != 0         # a window above the state
    assert call(12, 10, 11, 64)[0] != 0        # a chunk above the window
    assert call(12, 10, 3, 64)[0] != 0         # a chunk below 2^4 amplitudes
    assert call(41, 12, 0, 64)[0] != 0         # more than 40 qubits
    assert call(12, 12, 0, 64) == (0, 3 + 3 * 1)  # the whole state: one pass
    rc, need = call(12, 10, 8, 0)              # capacity 0: refused, size reported
    assert rc != 0 and need > 3
    out = (C.c_uint64 * need)()
    assert call(12, 10, 8, need) == (0, need)
    del keep
