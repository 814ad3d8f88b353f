"""Gate fusion wider than the reference's containment rule (fusion_width
2..6): the plan keeps the reference's structure (a gate joins the newest
open block sharing a qubit, blocks run in opening order), so the
reference's own block sweep (engines::dense::apply_blocks with the dense
engine's apply_matrix, through oracle/_ref) accepts it.  On the CPU: every
block is at most `width` wide, every operation lands in exactly one block,
and the fused run equals the unfused oracle within 1e-12 (a reordering of
exact arithmetic only).  On the GPU: the engine with the same width is
bitwise the reference's sweep of the same plan."""
import numpy as np
import pytest

from menos_b200 import workloads
from menos_b200.engine import fusion_plan
from test_host import as_oracle_circuit
from test_oracle_pin import random_circuit

WIDTHS = [2, 3, 4, 5, 6]


def circuits():
    rng = np.random.default_rng(5)
    yield "brick", workloads.brick(10, 8, 3)
    yield "brick+qft", workloads.qft(9, workloads.brick(9, 3, 4))
    yield "hea", workloads.hea(10, 4, 6)
    yield "random", random_circuit(9, 90, rng)


@pytest.mark.parametrize("width", WIDTHS)
def test_plan_shape_and_soundness(ref, oracle, width):
    for name, c in circuits():
        order, bb, bq, qb = fusion_plan(c, width)
        assert sorted(order.tolist()) == list(range(len(c.ops))), name
        for b in range(len(bb) - 1):
            # A block spans at most `width` qubits, or its one gate when that
            # gate alone is wider; its operands cover its members' qubits.
            qs = set(bq[qb[b]:qb[b + 1]].tolist())
            members = order[bb[b]:bb[b + 1]]
            widest = max(len(c.ops[i][1]) for i in members)
            assert len(qs) <= max(width, widest) and (len(qs) <= width or len(members) == 1), name
            for i in members:
                if c.ops[i][0] != 22:  # MeasureOps are barriers with no operands
                    assert set(c.ops[i][1]) <= qs, name
        fused = ref.run_plan(as_oracle_circuit(c), (order, bb, bq, qb))
        plain = oracle.run(as_oracle_circuit(c), fuse_gates=False)
        assert np.max(np.abs(fused - plain)) <= 1e-12, name


def test_width_zero_is_the_reference_containment_plan(ref):
    for name, c in circuits():
        order, bb, bq, qb = fusion_plan(c, 0)
        r = ref.plan_fusion(as_oracle_circuit(c))
        assert np.array_equal(order, r[0]) and np.array_equal(bb, r[1]), name
        assert np.array_equal(bq, r[2]) and np.array_equal(qb, r[3]), name


@pytest.mark.gpu
@pytest.mark.parametrize("width", [3, 4, 5])
def test_engine_bitwise_with_the_reference_sweep_of_the_same_plan(ctx, ref, width):
    from menos_b200 import DeviceState
    from test_oracle_pin import bits_equal
    cs = list(circuits()) + [("brick16", workloads.qft(16, workloads.brick(16, 6, 8)))]
    for name, c in cs:
        plan = fusion_plan(c, width)
        expect = ref.run_plan(as_oracle_circuit(c), plan)
        for tile in (0, 12):
            st = DeviceState(ctx, c.num_qubits)
            st.init(c.global_phase)
            st.apply_program(c, tile_qubits=tile, fusion_width=width)
            assert bits_equal(st.copy_out(), expect), (name, width, tile)
