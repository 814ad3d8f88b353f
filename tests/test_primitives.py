"""The Qiskit-shaped primitives (menos_b200/primitives.py).

CPU: Pauli labels and observables are read as the reference's
convert_observable reads a SparsePauliOp (bit j = qubit j, the label's last
character qubit 0, P = i^{|x&z|} X^x Z^z), and parameter binding fills the
parameterised gates' slots in op order.

GPU: every observable of a pub from one state equals the oracle's
expectation of the bound circuit; a parameterised pub's bindings (batched
sweep) equal their circuits run one by one; the result shape broadcasts the
bindings against the observables; the sampler's counts are the engine's for
the same seed and are keyed by Qiskit-ordered bitstrings.
"""
import types

import numpy as np
import pytest

from menos_b200 import workloads
from menos_b200.circuit import OP, Circuit
from menos_b200.primitives import bind, label_masks, observable_terms, parameter_slots


def test_label_masks_follow_qiskit_order():
    assert label_masks("I") == (0, 0)
    assert label_masks("XZ") == (0b10, 0b01)      # qubit 0 = Z, qubit 1 = X
    assert label_masks("YII") == (0b100, 0b100)
    with pytest.raises(ValueError):
        label_masks("XQ")


def test_observable_forms_agree():
    sp = types.SimpleNamespace(paulis=types.SimpleNamespace(x=[[0, 1, 0], [1, 1, 0]], z=[[1, 0, 0], [1, 0, 1]]),
                               coeffs=[0.5, -2.0 + 1j])
    a = observable_terms(sp, 3)
    b = observable_terms({"IXZ": 0.5, "ZXY": -2.0 + 1j}, 3)
    c = observable_terms([(0b010, 0b001, 0.5), (0b011, 0b101, -2.0 + 1j)], 3)
    assert a == b == c
    with pytest.raises(ValueError):
        observable_terms({"XIII": 1.0}, 3)


def test_bind_fills_parameter_slots_in_op_order():
    c = Circuit(2).gate("h", [0]).gate("rx", [0], [0.0]).gate("u", [1], [0, 0, 0]).gate("cx", [0, 1])
    c.gate("rzz", [0, 1], [0.0])
    assert parameter_slots(c) == 5
    b = bind(c, [1, 2, 3, 4, 5])
    assert [ps for _, _, ps, _, _ in b.ops] == [(), (1.0,), (2.0, 3.0, 4.0), (), (5.0,)]
    with pytest.raises(ValueError):
        bind(c, [1, 2])


@pytest.mark.gpu
def test_estimator_observables_from_one_state(ctx, oracle):
    from menos_b200.primitives import B200Estimator
    from test_host import as_oracle_circuit
    n = 12
    circ = workloads.brick(n, 6, 4)
    obs = [{"Z" + "I" * (n - 1): 1.0}, {"XX" + "I" * (n - 2): 0.5, "Y" * n: -1.5}, "IZ" * (n // 2)]
    est = B200Estimator(ctx, seed=1)
    (r,) = est.run([(circ, obs)])
    psi = oracle.run(as_oracle_circuit(circ))
    for i, o in enumerate(obs):
        want = sum((c * oracle.expectation(psi, x, z)).real for x, z, c in observable_terms(o, n))
        assert abs(r["evs"][i] - want) < 1e-12
    assert r["shape"] == (3,) and np.all(r["stds"] == 0)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [10, 18])
def test_estimator_parameter_bindings(ctx, n):
    from menos_b200 import DeviceState
    from menos_b200.primitives import B200Estimator
    circ = workloads.hea(n, 3, 7)
    p = parameter_slots(circ)
    values = np.random.default_rng(n).uniform(-np.pi, np.pi, size=(2, 3, p))
    obs = [["Z" + "I" * (n - 1)], [{"X" * n: 0.7, "IZ" * (n // 2): 0.2}]]  # shape (2, 1)
    (r,) = B200Estimator(ctx).run([(circ, obs, values)])
    assert r["shape"] == (2, 3)
    for i in range(2):
        for j in range(3):
            st = DeviceState(ctx, n)
            st.init(0.0)
            st.apply_program(bind(circ, values[i, j]))
            terms = observable_terms(obs[i][0], n)
            vals = st.expectation([(x, z) for x, z, _ in terms])
            want = sum((c * v).real for (_, _, c), v in zip(terms, vals))
            assert abs(r["evs"][i, j] - want) < 1e-12


@pytest.mark.gpu
def test_sampler_counts_are_the_engines(ctx):
    from menos_b200 import DeviceState
    from menos_b200.primitives import B200Sampler
    n = 10
    circ = workloads.brick(n, 5, 2)
    for q in range(n):
        circ.measure(q, q)
    smp = B200Sampler(ctx, seed=5)
    (r,) = smp.run([(circ,)], shots=3000)
    assert sum(r["counts"].values()) == 3000
    assert all(len(k) == n for k in r["counts"])
    # The same request alone through the engine, with the seed the sampler drew.
    seed = int(np.random.default_rng(5).integers(0, 2 ** 63))
    st = DeviceState(ctx, n)
    st.init(circ.global_phase)
    st.apply_program(circ)
    direct = st.sample(3000, seed, circ.measure_targets())
    assert r["counts"] == {format(k, f"0{n}b"): v for k, v in direct.items()}
    hea = workloads.hea(8, 2, 3)
    for q in range(8):
        hea.measure(q, q)
    vals = np.random.default_rng(0).uniform(-1, 1, size=(4, parameter_slots(hea)))
    (rb,) = smp.run([(hea, vals, 500)])
    assert rb["shape"] == (4,) and all(sum(c.values()) == 500 for c in rb["counts"])
    smp.close()
