"""The benchmarked workloads at their own sizes, against the reference.

* The 30-qubit complex128 job (a 16 GiB state: U3/CZ brick depth 40 + QFT,
  the bench's step): its 1e6-shot counts (seed 1234) equal the reference
  sampler's on the GPU's final state, and its 64 Pauli expectations agree
  with the reference's sequential per-term sum within 1e-12; a shortened
  30-qubit circuit with every gate kind of the job (U3, CZ, H, CP, SWAP on
  all qubit positions) is bitwise the reference's DenseEngine::execute.
* The complex64 precision workload (U3/CZ brick depth 32) at 28 qubits: the
  amplitude error and the error of 64 Pauli expectations against the FP64
  state -- the complex128 path, itself bitwise the reference -- within the
  precision path's bars (|d amp| <= 1e-6, |d<P>| <= 1e-6), and the same at
  24 qubits directly against the reference's own statevector.

The reference side runs in oracle/_ref (the reference's CPU sources), on the
host: these tests need the state twice or three times in host memory."""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from menos_b200 import DeviceState, workloads
from menos_b200.engine import C64
from test_host import as_oracle_circuit
from test_oracle_pin import bits_equal

pytestmark = pytest.mark.gpu

GIB = 1 << 30


def need_host_gib(gib):
    import psutil
    avail = psutil.virtual_memory().available
    if avail < gib * GIB:
        pytest.skip(f"needs {gib} GiB of free host memory, {avail / GIB:.0f} GiB free")


@pytest.fixture(scope="module")
def c2_host(ctx):
    """The job's final state: computed on the GPU, with the GPU's outputs,
    then copied to the host for the reference."""
    need_host_gib(40)
    n = 30
    st = DeviceState(ctx, n)
    st.init(0.0)
    st.apply_program(workloads.config_c2(n=n, depth=40))
    paulis = workloads.pauli_strings(n, 64, 7)
    out = {
        "counts": st.sample(10 ** 6, 1234, [(q, q) for q in range(n)]).to_dict(),
        "paulis": paulis,
        "terms": st.expectation(paulis),
        "norm": st.norm(),
        "amps": st.copy_out(),
    }
    st.free()
    yield out
    out.clear()


def test_c2_counts_identical_at_30_qubits(c2_host, ref):
    expect = ref.sample(c2_host["amps"], 10 ** 6, 1234, [(q, q) for q in range(30)], width=30)
    assert c2_host["counts"] == expect


def test_c2_pauli_expectations_at_30_qubits(c2_host, ref):
    amps = c2_host["amps"]
    with ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as ex:
        expect = list(ex.map(lambda p: ref.expectation(amps, p[0], p[1]), c2_host["paulis"]))
    got = c2_host["terms"]
    assert np.max(np.abs(np.asarray(expect) - got)) <= 1e-12
    # The norm is the one sum near 1.0: there the reference's strictly
    # sequential sum of 2^30 terms carries a few 1e-12 of rounding (about
    # sqrt(2^30) roundings of 1.1e-16), so both are held against a pairwise
    # sum of the same squares (error ~1e-15): the device's fixed-grid
    # reduction within 1e-13, the reference within 1e-11.
    pairwise = 0.0
    for i in range(0, amps.size, 1 << 24):
        chunk = amps[i:i + (1 << 24)]
        pairwise += float(np.sum(chunk.real * chunk.real + chunk.imag * chunk.imag))
    assert abs(c2_host["norm"] - pairwise) <= 1e-13
    assert abs(ref.expectation(amps, 0, 0).real - pairwise) <= 1e-11


def shortened_c2(n=30, seed=20260929):
    """Two brick layers, then the QFT's first two rows (H, every CP) and its
    final swaps: each of the job's gate kinds on every qubit position."""
    c = workloads.brick(n, 2, seed)
    two_pi = 2.0 * np.pi
    for j in range(2):
        c.gate("h", [j])
        for k in range(j + 1, n):
            c.gate("cp", [k, j], [two_pi / float(1 << (k - j + 1))])
    for i in range(n // 2):
        c.gate("swap", [i, n - 1 - i])
    return c


def test_c2_shortened_statevector_bitwise_at_30_qubits(ctx, ref):
    need_host_gib(56)
    c = shortened_c2()
    st = DeviceState(ctx, 30)
    st.init(0.0)
    st.apply_program(c)
    got = st.copy_out()
    st.free()
    expect = ref.run(as_oracle_circuit(c), fuse_gates=True)["statevector"]
    assert bits_equal(got, expect)


def c64_errors(ctx, n, depth, hi_amps, paulis):
    st = DeviceState(ctx, n, precision=C64)
    st.init(0.0)
    st.apply_program(workloads.brick(n, depth, 20260929))
    st.normalize()
    terms = st.expectation(paulis)
    lo = st.copy_out()
    st.free()
    amp_err = float(np.max(np.abs(lo.astype(np.complex128) - hi_amps)))
    return amp_err, terms


def test_c64_error_at_28_qubits(ctx):
    need_host_gib(16)
    n, depth = 28, 32
    paulis = workloads.pauli_strings(n, 64, 21)
    hi = DeviceState(ctx, n)
    hi.init(0.0)
    hi.apply_program(workloads.brick(n, depth, 20260929))
    hi_terms = hi.expectation(paulis)
    hi_amps = hi.copy_out()
    hi.free()
    amp_err, terms = c64_errors(ctx, n, depth, hi_amps, paulis)
    assert amp_err <= 1e-6
    assert np.max(np.abs(terms - hi_terms)) <= 1e-6


def test_c64_error_at_24_qubits_against_reference(ctx, ref):
    n, depth = 24, 32
    paulis = workloads.pauli_strings(n, 64, 21)
    r = ref.run(as_oracle_circuit(workloads.brick(n, depth, 20260929)), fuse_gates=True, paulis=paulis)
    amp_err, terms = c64_errors(ctx, n, depth, r["statevector"], paulis)
    assert amp_err <= 1e-6
    assert np.max(np.abs(terms - r["terms"])) <= 1e-6
