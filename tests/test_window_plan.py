"""The window plan of the chunked tier on the copy engines
(mb2_window_plan, what mb2_apply_program_windowed runs) against the
reference's own pass planner compiled from its sources
(src/engines/dense_tiered/pass_plan.cpp: build_pass_plan's greedy rule over
the fusion plan's blocks, choose_pass_plan's chunk choice)."""
import ctypes as C

import numpy as np
import pytest

import pyoracle
from menos_b200 import workloads
from menos_b200._lib import SweepOptions, lib
from menos_b200.circuit import to_mb2_ops
from test_oracle_pin import random_circuit


def window_plan(circ, window, chunk):
    arr, keep = to_mb2_ops(circ)
    out = (C.c_uint64 * (1 << 18))()
    nw = C.c_uint64(1 << 18)
    opts = SweepOptions(1, 0, 0, 0, 0, 0)
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
