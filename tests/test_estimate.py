"""The sweep estimate (mb2_estimate_sweep: the dense work units of
DenseEngine::estimate, src/engines/dense/dense_engine.cpp:309-331) against
the hand-computed values of the reference's own tests
(tests/engines/dense/dense_engine_test.cpp:59-185).  The reference adds 2^n
per requested output (statevector, counts) above the sweep; the sweep's part
is 2^n for initialisation plus 2^(n+k) per block of k qubits.  Host only."""
import ctypes as C

import pytest

from menos_b200._lib import MB2Error, SweepEstimate, SweepOptions, lib
from menos_b200.circuit import Circuit, to_mb2_ops


def estimate(circ, fuse=True, n=None):
    arr, keep = to_mb2_ops(circ)
    out = SweepEstimate()
    opts = SweepOptions(1 if fuse else 0, 0, 0, 0, 0, 0)
    rc = lib().mb2_estimate_sweep(arr, len(circ.ops), C.byref(opts), circ.num_qubits if n is None else n,
                                  C.byref(out))
    del keep
    if rc != 0:
        raise MB2Error(rc, "mb2_estimate_sweep")
    return out


def bell():
    return Circuit(2).gate("h", [0]).gate("cx", [0, 1])


def test_hand_computable_unfused():
    # ExactHandComputableValueWithStatevector (:59-86): 4 (init) + 8 (H) + 16
    # (CX) + 4 (the statevector pass) = 32.
    e = estimate(bell(), fuse=False)
    assert e.blocks == 2
    assert e.work_units + 4 == 32


def test_fused_bell_is_one_block():
    # FusedBellIsOnePassAndChargesThePlanAndTheBlock (:88-109): one 2-qubit
    # block, 4 + 16 + 4.
    e = estimate(bell(), fuse=True)
    assert e.blocks == 1
    assert e.work_units + 4 == 4 + 16 + 4


def test_both_outputs_add_both_pass_terms():
    # BothOutputsRequestedAddsBothPassTerms (:134-141): 4 + 8 + 4 + 4 = 20.
    e = estimate(Circuit(2).gate("h", [0]), fuse=False)
    assert e.work_units + 4 + 4 == 20


def test_measure_contributes_no_work():
    # MeasureOpContributesNoPerOperationWork (:143-155).
    with_m = Circuit(2, 1).gate("h", [0])
    with_m.measure(0, 0)
    assert estimate(with_m, fuse=False).work_units == estimate(Circuit(2).gate("h", [0]), fuse=False).work_units


def test_empty_region_is_initialisation():
    # EmptyRegionIsJustInitialization (:157-164): 2^3.
    e = estimate(Circuit(3))
    assert (e.blocks, e.work_units, e.passes) == (0, 8, 0)
    assert e.device_bytes == 16 * 8


def test_sizes_past_the_device_are_refused():
    # The reference marks 2^62 and 2^63 work infeasible (:166-185); a state
    # above 2^40 amplitudes (16 TiB) is refused here before any arithmetic.
    with pytest.raises(MB2Error):
        estimate(Circuit(2).gate("cx", [0, 1]), n=62)
    with pytest.raises(MB2Error):
        estimate(Circuit(1), n=63)
    assert estimate(Circuit(2).gate("cx", [0, 1]), fuse=False, n=40).work_units == (1 << 40) + (1 << 42)
