"""The complex64 precision path against the FP64 oracle: amplitude and
expectation errors stay at FP32 rounding scale, and its sampler reproduces
the reference walk over the state's own (FP64-promoted) probabilities."""
import numpy as np
import pytest

from menos_b200 import DeviceState, workloads
from menos_b200._lib import C64
from test_host import as_oracle_circuit
from test_oracle_pin import random_circuit

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kernel", ["tensor", "simt"])
@pytest.mark.parametrize("n", [4, 7, 11, 14])
def test_c64_random_circuits_within_fp32_error(ctx, oracle, n, kernel):
    rng = np.random.default_rng(n)
    for fuse in (True, False):
        c = random_circuit(n, 120, rng)
        st = DeviceState(ctx, n, precision=C64)
        st.init(c.global_phase)
        st.apply_program(c, fuse_gates=fuse, c64_kernel=kernel)
        got = st.copy_out().astype(np.complex128)
        expect = oracle.run(as_oracle_circuit(c), fuse_gates=fuse)
        assert np.max(np.abs(got - expect)) < 2e-5, (n, fuse)
        terms = [(int(rng.integers(0, 1 << n)), int(rng.integers(0, 1 << n))) for _ in range(8)]
        e = st.expectation(terms)
        for (x, z), v in zip(terms, e):
            assert abs(v - oracle.expectation(expect, x, z)) < 2e-5


def test_c64_brick_error_and_renormalisation(ctx, ref):
    n = 20
    c = workloads.brick(n, 16, 77)
    st = DeviceState(ctx, n, precision=C64)
    st.init(0.0)
    st.apply_program(c)
    before = st.normalize()
    assert abs(before - 1.0) < 1e-4
    assert abs(st.norm() - 1.0) < 1e-6
    got = st.copy_out().astype(np.complex128)
    expect = ref.run(as_oracle_circuit(c))["statevector"]
    assert np.max(np.abs(got - expect)) < 1e-5
    paulis = workloads.pauli_strings(n, 16, 3)
    r = ref.run(as_oracle_circuit(c), statevector=False, paulis=paulis)
    assert np.max(np.abs(st.expectation(paulis) - r["terms"])) < 1e-6


def test_c64_sampler_walks_the_promoted_state(ctx, oracle):
    n = 16
    c = workloads.brick(n, 6, 5)
    st = DeviceState(ctx, n, precision=C64)
    st.init(0.0)
    st.apply_program(c)
    promoted = st.copy_out().astype(np.complex128)
    t = [(q, q) for q in range(n)]
    assert st.sample(20000, 3, t) == oracle.sample(promoted, 20000, 3, t)
