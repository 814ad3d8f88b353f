"""The reference's own CUDA dense engine (CudaDenseEngine, src/kernels/cuda
built for sm_100a with its -fmad=false by oracle/Makefile) beside this
engine: both are bitwise the reference CPU engine's statevector, give its
counts and agree on Pauli terms -- so the GPU "before" number that
bench.py --impl reference reports is timed on the same results."""
import os

import numpy as np
import pytest

import pyoracle
from test_host import as_oracle_circuit
from test_oracle_pin import random_circuit

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refcuda():
    if not os.path.exists(pyoracle.REF_CUDA_SO):
        pytest.skip("reference CUDA library not built (oracle/_ref)")
    return pyoracle.RefLib(pyoracle.REF_CUDA_SO)


@pytest.mark.parametrize("fuse", [True, False])
def test_reference_cuda_engine_matches_cpu_and_this_engine(ctx, refcuda, fuse):
    from menos_b200 import DeviceState
    n = 16
    c = random_circuit(n, 200, np.random.default_rng(11 if fuse else 12))
    oc = as_oracle_circuit(c)
    t = [(q, q) for q in range(n)]
    paulis = [(int(x), int(z)) for x, z in np.random.default_rng(5).integers(0, 1 << n, size=(8, 2))]
    cpu = refcuda.run(oc, fuse_gates=fuse, threads=1, shots=5000, seed=9, targets=t, paulis=paulis)
    gpu = refcuda.run(oc, fuse_gates=fuse, shots=5000, seed=9, targets=t, paulis=paulis, engine="cuda")
    assert np.array_equal(cpu["statevector"].view(np.uint64), gpu["statevector"].view(np.uint64))
    assert cpu["counts"] == gpu["counts"]
    st = DeviceState(ctx, n)
    st.init(c.global_phase)
    st.apply_program(c, fuse_gates=fuse)
    assert np.array_equal(st.copy_out().view(np.uint64), cpu["statevector"].view(np.uint64))
    assert np.max(np.abs(st.expectation(paulis) - gpu["terms"])) < 1e-12
