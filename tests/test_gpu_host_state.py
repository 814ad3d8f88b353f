"""Host-resident states (mb2_state_alloc_host): a complex128 state in pinned,
mapped host memory, swept by the same kernels over PCIe, gives the
device-resident state's results bit for bit -- amplitudes, counts, Pauli
terms and the exact norm -- and is refused over its host budget before any
allocation."""
import numpy as np
import pytest

from menos_b200 import DeviceState, workloads
from menos_b200._lib import ResourceExceeded
from test_oracle_pin import random_circuit

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [9, 17, 22])
def test_host_state_is_bitwise_the_device_state(ctx, n):
    circs = [workloads.config_c2(n=n, depth=6), random_circuit(n, 150, np.random.default_rng(n))]
    paulis = workloads.pauli_strings(n, 12, 5)
    t = [(q, q) for q in range(n)]
    for c in circs:
        out = []
        for host in (False, True):
            st = DeviceState(ctx, n, host=host)
            st.init(c.global_phase)
            st.apply_program(c)
            out.append((st.copy_out(), st.sample(20000, 7, t).to_dict(), st.expectation(paulis), st.norm_exact()))
            st.free()
        (a0, c0, e0, n0), (a1, c1, e1, n1) = out
        assert np.array_equal(a0.view(np.uint64), a1.view(np.uint64))
        assert c0 == c1 and n0 == n1
        assert np.array_equal(e0.view(np.uint64), e1.view(np.uint64))


def test_host_state_budget_is_checked_first(ctx):
    with pytest.raises(ResourceExceeded):
        DeviceState(ctx, 24, host=True, budget_bytes=(16 << 24) - 1)


@pytest.mark.parametrize("n,window,chunk", [(20, 16, 12), (20, 14, 8), (20, 12, 0), (20, 20, 20), (18, 17, 0)])
def test_windowed_sweep_is_bitwise_the_device_state(ctx, n, window, chunk):
    """The chunked tier on the copy engines: windows of 2^window amplitudes
    (chunks of 2^chunk; 0: chosen), double-buffered, the blocks remapped."""
    circs = [workloads.config_c2(n=n, depth=8), random_circuit(n, 200, np.random.default_rng(100 + n))]
    for c in circs:
        dev = DeviceState(ctx, n)
        dev.init(c.global_phase)
        dev.apply_program(c)
        want = dev.copy_out()
        dev.free()
        st = DeviceState(ctx, n, host=True)
        st.init(c.global_phase)
        stats = st.apply_program_windowed(c, window, chunk)
        got = st.copy_out()
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
        assert stats.passes >= 1 and stats.blocks > 0
        # Outputs read the swept host state as before.
        assert st.sample(5000, 3, [(q, q) for q in range(n)]).to_dict() == \
            _device_counts(ctx, c, n, 5000, 3)
        st.free()


def _device_counts(ctx, c, n, shots, seed):
    st = DeviceState(ctx, n)
    st.init(c.global_phase)
    st.apply_program(c)
    out = st.sample(shots, seed, [(q, q) for q in range(n)]).to_dict()
    st.free()
    return out


def test_windowed_sweep_refusals(ctx):
    from menos_b200._lib import MB2Error
    n = 14
    c = workloads.config_c2(n=n, depth=3)
    dev = DeviceState(ctx, n)
    dev.init()
    with pytest.raises(MB2Error, match="host-resident"):
        dev.apply_program_windowed(c, 12, 8)
    st = DeviceState(ctx, n, host=True)
    st.init()
    # Chunks as large as the window leave no room for a block's upper operands.
    with pytest.raises(MB2Error, match="window"):
        st.apply_program_windowed(c, 10, 10)
