"""mb2_expectation_noalloc: the Pauli-expectation reduction for callers that
cannot allocate device memory (a process whose own allocator holds the GPU's
memory, or code that must not enter the driver's allocator).  Its scratch is
a fixed file-scope device array instead of a cudaMalloc.

Called through the C ABI on a state this test allocates with the ordinary
API, twice in a row with different terms, and checked against
mb2_expectation's output with the parity tests' tolerance.  Runs last in the
suite (file name) and passes alone in a fresh process too."""
import ctypes as C

import numpy as np
import pytest

from menos_b200 import DeviceState, workloads
from menos_b200._lib import lib

pytestmark = pytest.mark.gpu

EXP_TOL = 1e-12
MAX_TERMS = 64


def noalloc(st, terms):
    xs = np.ascontiguousarray([t[0] for t in terms], dtype=np.uint64)
    zs = np.ascontiguousarray([t[1] for t in terms], dtype=np.uint64)
    out = np.zeros(2 * len(terms), np.float64)
    dev = C.c_void_p()
    assert lib().mb2_state_device_ptr(st.h, C.byref(dev)) == 0
    st.synchronize()
    rc = lib().mb2_expectation_noalloc(dev, st.n, xs.ctypes.data, zs.ctypes.data, len(terms), out.ctypes.data,
                                       C.c_void_p(st.stream_handle()))
    return rc, out.view(np.complex128)


def test_noalloc_expectation_matches_the_allocating_entry_point(ctx):
    n = 18
    c = workloads.brick(n, 6, 5)
    st = DeviceState(ctx, n)
    st.init(0.3)
    st.apply_program(c)
    first = [(0, 0)] + workloads.pauli_strings(n, MAX_TERMS - 1, 11)
    second = workloads.pauli_strings(n, 17, 12)
    for terms in (first, second):
        rc, got = noalloc(st, terms)
        assert rc == 0
        expect = st.expectation(terms)
        assert np.max(np.abs(got - expect)) <= EXP_TOL


def test_noalloc_rejects_more_terms_than_its_scratch_holds(ctx):
    st = DeviceState(ctx, 6)
    st.init(0.0)
    rc, _ = noalloc(st, [(1, 0)] * (MAX_TERMS + 1))
    assert rc == 2  # MB2_ERR_RESOURCE
