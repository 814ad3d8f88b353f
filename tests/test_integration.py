"""The reference-side binding (menos_b200/integration/b200_dense_engine.cpp,
a menos::SimulationEngine over the C ABI) compiles against the reference's
own headers.  CPU only; skipped where the reference sources are absent."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

REF = os.environ.get("MENOS_REFERENCE_ROOT", "/root/reference")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "include", "menos")), reason="reference headers absent")
def test_adapter_compiles_against_reference_headers():
    cxx = shutil.which("g++")
    assert cxx
    src = os.path.join(ROOT, "menos_b200", "integration", "b200_dense_engine.cpp")
    r = subprocess.run([cxx, "-std=c++20", "-fsyntax-only", "-Wall", f"-I{REF}/include", f"-I{REF}/src",
                        f"-I{ROOT}/include", src], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
