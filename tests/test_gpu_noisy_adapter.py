"""The noisy engines' reference-side binding (menos_b200/integration/
b200_noisy_engines.cpp) run through menos::SimulationEngine::execute beside
the reference's own DensityMatrixEngine and TrajectoryEngine, linked in one
library (oracle/_ref/libmenos_adapter.so): identical counts (readout errors
included), identical Factorized draws, traces and term means within 1e-12,
the same standard error, the monitor's safe boundaries, the Device-space
ledger charge and the reference's refusals."""
import numpy as np
import pytest

import pyadapter
from test_dm import noisy_circuit, with_readout_measures
from test_trajectories import pure_noise_circuit

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def harness():
    return pyadapter.AdapterHarness()


@pytest.mark.parametrize("n", [2, 5])
def test_dm_binding_is_the_reference_engine(harness, n):
    rng = np.random.default_rng(700 + n)
    c, _ = noisy_circuit(n, 30, rng)
    targets = with_readout_measures([c], n, rng)
    paulis = [(int(rng.integers(0, 1 << n)), int(rng.integers(0, 1 << n))) for _ in range(10)] + [(0, 0)]
    kw = dict(shots=20000, seed=21, targets=targets, paulis=paulis)
    ref = harness.execute(pyadapter.REFERENCE_DM, c, **kw)
    got = harness.execute(pyadapter.B200_DM, c, **kw)
    assert ref["rc"] == got["rc"] == pyadapter.OK, got["error"]
    assert got["counts"] == ref["counts"]
    assert np.max(np.abs(got["terms"] - ref["terms"])) < 1e-12
    assert got["peak_device"] == 16 << (2 * n)
    assert harness.estimate(pyadapter.B200_DM, c, **kw)["work_units"] == \
        harness.estimate(pyadapter.REFERENCE_DM, c, **kw)["work_units"]


def test_dm_binding_factorized_draws(harness):
    n = 4
    rng = np.random.default_rng(711)
    c, _ = noisy_circuit(n, 24, rng)
    targets = with_readout_measures([c], n, rng)
    kw = dict(shots=3000, seed=5, targets=targets, sole=False, draws=3000, draw_seed=99)
    ref = harness.execute(pyadapter.REFERENCE_DM, c, **kw)
    got = harness.execute(pyadapter.B200_DM, c, **kw)
    assert ref["has_sampler"] and got["has_sampler"]
    assert np.array_equal(got["drawn"], ref["drawn"])


def test_dm_binding_monitor_and_refusals(harness):
    n = 3
    c, _ = noisy_circuit(n, 20, np.random.default_rng(712))
    ref = harness.execute(pyadapter.REFERENCE_DM, c, shots=10, targets=[(0, 0)], abandon_at=7)
    got = harness.execute(pyadapter.B200_DM, c, shots=10, targets=[(0, 0)], abandon_at=7)
    assert ref["rc"] == got["rc"] == pyadapter.INTERNAL_ERROR
    assert got["monitor_calls"] == ref["monitor_calls"] == 7
    est = harness.estimate(pyadapter.B200_DM, c, statevector=True)
    assert not est["feasible"] and "statevector" in est["reason"]


@pytest.mark.parametrize("n", [3, 9])
def test_trajectory_binding_is_the_reference_engine(harness, n):
    c = pure_noise_circuit(n, 30, 720 + n, widest=3)
    targets = with_readout_measures([c], n, np.random.default_rng(n))
    rng = np.random.default_rng(730 + n)
    paulis = [(int(x), int(z)) for x, z in rng.integers(0, 1 << n, size=(6, 2))] + [(0, 0)]
    coefs = rng.normal(size=len(paulis)) + 1j * rng.normal(size=len(paulis))
    kw = dict(shots=64, seed=2026, targets=targets, paulis=paulis, coefs=coefs, trajectories=80)
    ref = harness.execute(pyadapter.REFERENCE_TRAJ, c, **kw)
    got = harness.execute(pyadapter.B200_TRAJ, c, **kw)
    assert ref["rc"] == got["rc"] == pyadapter.OK, got["error"]
    assert got["statistical"] and ref["statistical"]
    assert got["counts"] == ref["counts"]
    assert np.max(np.abs(got["terms"] - ref["terms"])) < 1e-12
    assert abs(got["standard_error"] - ref["standard_error"]) <= 1e-9 * max(1.0, ref["standard_error"])
    assert got["peak_device"] == 16 << n
    assert harness.estimate(pyadapter.B200_TRAJ, c, **kw)["work_units"] == \
        harness.estimate(pyadapter.REFERENCE_TRAJ, c, **kw)["work_units"]


def test_trajectory_binding_monitor_and_refusals(harness):
    n = 3
    c = pure_noise_circuit(n, 12, 740, widest=2)
    per = len(c.ops) + 1
    # Abandoned on the third trajectory's end boundary: both engines stop there.
    ref = harness.execute(pyadapter.REFERENCE_TRAJ, c, paulis=[(1, 0)], trajectories=10, abandon_at=3 * per)
    got = harness.execute(pyadapter.B200_TRAJ, c, paulis=[(1, 0)], trajectories=10, abandon_at=3 * per)
    assert ref["rc"] == got["rc"] == pyadapter.INTERNAL_ERROR
    # Not a sole region; more shots than trajectories: refused as the reference refuses.
    for kw in (dict(sole=False, shots=4, targets=[(0, 0)], trajectories=8),
               dict(shots=9, targets=[(0, 0)], trajectories=8)):
        assert harness.execute(pyadapter.REFERENCE_TRAJ, c, **kw)["rc"] == pyadapter.INTERNAL_ERROR
        assert harness.execute(pyadapter.B200_TRAJ, c, **kw)["rc"] == pyadapter.INTERNAL_ERROR
