"""The reference-side binding (menos_b200/integration/b200_dense_engine.cpp,
the menos::SimulationEngine MENOS would register) on the CPU: it compiles
against the reference's headers, and the library oracle/Makefile links from
it, the reference's CPU engine objects and libmenos_b200.so loads, exports
its harness and, with no device present, answers as the reference's CUDA
engine does without one (estimate infeasible, execute refused with
InternalError).  The GPU differential cases are tests/test_gpu_adapter.py."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

REF = os.environ.get("MENOS_REFERENCE_ROOT", "")
ADAPTER_SO = os.path.join(ROOT, "oracle", "_ref", "libmenos_adapter.so")


@pytest.mark.skipif(not (REF and os.path.isdir(os.path.join(REF, "include", "menos"))),
                    reason="MENOS_REFERENCE_ROOT does not name the reference sources")
def test_adapter_compiles_against_reference_headers():
    cxx = shutil.which("g++")
    assert cxx
    src = os.path.join(ROOT, "menos_b200", "integration", "b200_dense_engine.cpp")
    r = subprocess.run([cxx, "-std=c++20", "-fsyntax-only", "-Wall", "-Wextra", f"-I{REF}/include", f"-I{REF}/src",
                        f"-I{ROOT}/include", src], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.skipif(not (REF and os.path.isdir(os.path.join(REF, "include", "menos"))),
                    reason="MENOS_REFERENCE_ROOT does not name the reference sources")
def test_noisy_adapters_compile_against_reference_headers():
    cxx = shutil.which("g++")
    assert cxx
    src = os.path.join(ROOT, "menos_b200", "integration", "b200_noisy_engines.cpp")
    r = subprocess.run([cxx, "-std=c++20", "-fsyntax-only", "-Wall", "-Wextra", f"-I{REF}/include", f"-I{REF}/src",
                        f"-I{ROOT}/include", src], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.skipif(not os.path.exists(ADAPTER_SO), reason="adapter library not built (oracle/_ref)")
def test_noisy_adapters_without_device():
    """The density-matrix and trajectory bindings answer as the dense one
    does without a device, while the reference's own engines in the same
    library run."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present: tests/test_gpu_noisy_adapter.py covers the bindings")
    import numpy as np
    import pyadapter
    from pyoracle import Circuit
    h = pyadapter.AdapterHarness()
    c = Circuit(2).gate("h", [0]).gate("cx", [0, 1])
    c.channel([1], np.array([[[1, 0], [0, 0.8]], [[0, 0.6], [0, 0]]], np.complex128))
    for eng in (pyadapter.B200_DM, pyadapter.B200_TRAJ):
        est = h.estimate(eng, c, shots=10, targets=[(0, 0)], trajectories=10)
        assert not est["feasible"] and "no B200 device" in est["reason"]
        r = h.execute(eng, c, shots=10, targets=[(0, 0)], trajectories=10)
        assert r["rc"] == pyadapter.INTERNAL_ERROR and "no device" in r["error"]
    ref = h.execute(pyadapter.REFERENCE_DM, c, shots=100, seed=1, targets=[(0, 0), (1, 1)])
    assert ref["rc"] == pyadapter.OK and sum(ref["counts"].values()) == 100
    tr = h.execute(pyadapter.REFERENCE_TRAJ, c, paulis=[(0, 2)], trajectories=20)
    assert tr["rc"] == pyadapter.OK and tr["statistical"] and tr["standard_error"] is not None


@pytest.mark.skipif(not os.path.exists(ADAPTER_SO), reason="adapter library not built (oracle/_ref)")
def test_adapter_library_links_and_runs_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present: tests/test_gpu_adapter.py covers the adapter")
    import pyadapter
    from pyoracle import Circuit
    h = pyadapter.AdapterHarness()
    c = Circuit(3).gate("h", [0]).gate("cx", [0, 1])
    est = h.estimate(pyadapter.B200, c, statevector=True)
    assert not est["feasible"] and "no B200 device" in est["reason"]
    r = h.execute(pyadapter.B200, c, statevector=True)
    assert r["rc"] == pyadapter.INTERNAL_ERROR and "no device" in r["error"]
    # The reference CPU engine in the same library still runs.
    ref = h.execute(pyadapter.REFERENCE_CPU, c, statevector=True)
    assert ref["rc"] == pyadapter.OK
    assert abs(ref["statevector"][0]) == pytest.approx(2 ** -0.5)
    assert h.calibration()["present"] == 0.0
