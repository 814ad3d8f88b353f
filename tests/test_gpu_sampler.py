"""The device sampler against the reference's sequential walk
(src/engines/dense/sample.cpp:24-75): identical counts, at sizes where the
chunked parity-map scan carries almost all of the walk, and on states built to
hit round-to-even ties and binade crossings."""
import numpy as np
import pytest

from menos_b200 import DeviceState, workloads
from test_gpu_parity import dev_state
from test_oracle_pin import rand_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [12, 17, 21, 23])
def test_random_states_identical_counts(ctx, oracle, n):
    rng = np.random.default_rng(n)
    s = rand_state(n, rng)
    st = dev_state(ctx, s)
    t = [(q, q) for q in range(n)]
    for shots, seed in [(4096, 1), (200000, 99)]:
        assert st.sample(shots, seed, t) == oracle.sample(s, shots, seed, t), (n, shots)


def test_skewed_magnitudes(ctx, oracle):
    # Amplitudes spanning many binades: most chunks sit in small binades early.
    n = 20
    rng = np.random.default_rng(3)
    mag = np.exp(rng.uniform(-30, 0, size=1 << n))
    s = (mag * np.exp(1j * rng.uniform(0, 6.3, size=1 << n))).astype(np.complex128)
    s /= np.linalg.norm(s)
    st = dev_state(ctx, s)
    t = [(q, q) for q in range(n)]
    assert st.sample(300000, 5, t) == oracle.sample(s, 300000, 5, t)


def test_round_to_even_ties(ctx, oracle):
    # |a|^2 = 2^-18 on even indices and 2^-54 on odd ones: once the running
    # sum reaches [0.5, 1) every odd element adds exactly half an ulp (a tie);
    # in [0.25, 0.5) it adds exactly one ulp.  Amplitudes are exact powers of two.
    n = 20
    s = np.zeros(1 << n, np.complex128)
    s[0::2] = 2.0 ** -9
    s[1::2] = 2.0 ** -27
    st = dev_state(ctx, s)
    t = [(q, q) for q in range(n)]
    for seed in (0, 1, 2):
        assert st.sample(100000, seed, t) == oracle.sample(s, 100000, seed, t)
    # and with imaginary parts carrying the weight
    s2 = s * 1j
    st2 = dev_state(ctx, s2)
    assert st2.sample(50000, 9, t) == oracle.sample(s2, 50000, 9, t)


def test_sparse_and_basis_states(ctx, oracle):
    n = 18
    for idx in (0, 1, (1 << n) - 1, 12345):
        s = np.zeros(1 << n, np.complex128)
        s[idx] = 1.0
        st = dev_state(ctx, s)
        t = [(q, q) for q in range(n)]
        assert st.sample(1000, 4, t) == oracle.sample(s, 1000, 4, t) == {idx: 1000}
    # total below one: the leftover shots go to the last basis state
    s = np.zeros(1 << n, np.complex128)
    s[5] = np.sqrt(0.3)
    st = dev_state(ctx, s)
    t = [(q, q) for q in range(n)]
    assert st.sample(5000, 8, t) == oracle.sample(s, 5000, 8, t)


def test_circuit_state_24_qubits(ctx, oracle):
    # A brick-circuit state at 24 qubits (4096 chunks), counts for 1e6 shots.
    n = 24
    c = workloads.brick(n, 4, 21)
    st = DeviceState(ctx, n)
    st.init(0.0)
    st.apply_program(c)
    s = st.copy_out()
    t = [(q, q) for q in range(n)]
    assert st.sample(1_000_000, 1234, t) == oracle.sample(s, 1_000_000, 1234, t)
