"""Grouped Pauli expectation on the GPU against the oracle: many terms that
share reads of the state (random strings, Z strings, X only in the low
bits, the identity, all-X / all-Z), complex128 and complex64 states, within
1e-12 absolute of the oracle's sequential sum (complex64: the promoted FP64
sum of the same amplitudes).  The value is reproducible bit for bit, and the
launches are one per shared group (one per term that shares nothing) plus
one finish."""
import ctypes as C

import numpy as np
import pytest

from menos_b200 import DeviceState, _lib
from menos_b200._lib import C64
from test_oracle_pin import rand_state
from test_pauli_groups import plan

pytestmark = pytest.mark.gpu

EXP_TOL = 1e-12


def term_mix(n, rng, count=64):
    full = (1 << n) - 1
    terms = [(0, 0), (full, 0), (0, full), (full, full)]
    terms += [(int(rng.integers(0, 1 << n)), int(rng.integers(0, 1 << n))) for _ in range(count)]
    terms += [(0, int(rng.integers(0, 1 << n))) for _ in range(8)]
    terms += [(int(rng.integers(1, 8)) & full, int(rng.integers(0, 1 << n))) for _ in range(8)]
    terms += [(1 << (n - 1), 1 << (n - 1)), (1, 0)]
    return terms


def launches():
    v = C.c_uint64()
    assert _lib.lib().mb2_kernel_launches(C.byref(v)) == 0
    return v.value


@pytest.mark.parametrize("n", [1, 4, 12, 13, 20])
def test_grouped_expectation_matches_oracle(ctx, oracle, n):
    rng = np.random.default_rng(100 + n)
    s = rand_state(n, rng)
    st = DeviceState(ctx, n)
    st.copy_in(s)
    terms = term_mix(n, rng)
    before = launches()
    got = st.expectation(terms)
    # One launch per shared group, one per term that shares nothing (or
    # whose state is below the grouped tiles' 2^10), one finish.
    expect = sum(1 if len(g[4]) > 1 and g[0] + g[1] >= 10 else len(g[4]) for g in plan(terms, n)) + 1
    assert launches() - before == expect
    for (x, z), g in zip(terms, got):
        e = oracle.expectation(s, x, z)
        assert abs(g - e) <= EXP_TOL, (n, x, z, g, e)
    again = st.expectation(terms)
    assert np.array_equal(got.view(np.uint64), again.view(np.uint64))


def test_grouped_expectation_complex64(ctx, oracle):
    rng = np.random.default_rng(7)
    n = 18
    s = rand_state(n, rng).astype(np.complex64)
    st = DeviceState(ctx, n, precision=C64)
    st.copy_in(s)
    terms = term_mix(n, rng, 40)
    got = st.expectation(terms)
    promoted = s.astype(np.complex128)
    for (x, z), g in zip(terms, got):
        e = oracle.expectation(promoted, x, z)
        assert abs(g - e) <= EXP_TOL, (x, z, g, e)
