"""Regenerates tests/golden/golden.json from the reference MENOS CPU engine
compiled from its own sources (oracle/_ref/libmenos_ref.so, built by
``make -C oracle ref`` where the reference sources are present).

    python tests/golden/make_golden.py

Every value is the reference's output: the mt19937_64 uniforms of
common::Rng, ir::generate_matrix for every named gate, and
DenseEngine::execute (statevector, counts, expectation terms) on small
seeded circuits.  Doubles are stored as float.hex strings (bit-exact).
"""
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle  # noqa: E402

OPS_1Q = ["x", "y", "z", "h", "s", "sdg", "t", "tdg", "sx", "sxdg", "rx", "ry", "rz", "p", "u"]
OPS_2Q = ["cx", "cz", "swap", "cp", "rzz"]
NPAR = {"rx": 1, "ry": 1, "rz": 1, "p": 1, "cp": 1, "rzz": 1, "u": 3}


def hexes(a):
    return [float.hex(float(x)) for x in np.asarray(a).view(np.float64).ravel()]


def circuit_ops(n, n_ops, seed):
    rng = np.random.default_rng(seed)
    ops = []
    for _ in range(n_ops):
        pool = OPS_1Q + (OPS_2Q if n >= 2 else []) + (["ccx"] if n >= 3 else [])
        name = pool[int(rng.integers(0, len(pool)))]
        nq = 3 if name == "ccx" else (2 if name in OPS_2Q else 1)
        qs = [int(q) for q in rng.permutation(n)[:nq]]
        ps = [float(p) for p in rng.uniform(-2 * math.pi, 2 * math.pi, size=NPAR.get(name, 0))]
        ops.append([name, qs, ps])
    return ops


def main():
    ref = pyoracle.RefLib()
    out = {"source": "reference MENOS CPU dense engine (oracle/_ref), see make_golden.py"}
    out["uniforms"] = [{"seed": s, "hex": [v.hex() for v in ref.uniforms(s, 16)]} for s in (42, 20260929)]
    gm = []
    for name in OPS_1Q + OPS_2Q + ["ccx"]:
        for params in ([0.0, 0.0, 0.0], [0.7, -1.9, 2.5], [-3.1, 4.4, 0.0001]):
            gm.append({"opcode": pyoracle.OP[name], "params": params[:NPAR.get(name, 0)],
                       "hex": hexes(ref.gate_matrix(pyoracle.OP[name], params))})
    out["gate_matrices"] = gm
    circuits = []
    for idx, (n, n_ops, fuse, gp) in enumerate([(1, 8, False, 0.0), (3, 30, True, 0.5), (5, 60, True, -1.25),
                                                (6, 80, False, 3.0), (8, 120, True, 0.0)]):
        ops = circuit_ops(n, n_ops, 1000 + idx)
        c = pyoracle.Circuit(n, gp)
        for name, qs, ps in ops:
            c.gate(name, qs, ps)
        paulis = [(int(x), int(z)) for x, z in np.random.default_rng(77 + idx).integers(0, 1 << n, size=(4, 2))]
        r = ref.run(c, fuse_gates=fuse, threads=1, statevector=True, shots=4096, seed=7 + idx,
                    targets=[(q, q) for q in range(n)], width=n, paulis=paulis)
        circuits.append({
            "name": f"random_n{n}", "n": n, "global_phase": gp, "fuse": fuse, "ops": ops,
            "statevector_hex": hexes(r["statevector"]), "shots": 4096, "seed": 7 + idx,
            "counts": {str(k): v for k, v in r["counts"].items()},
            "paulis": paulis, "terms": [[t.real.hex(), t.imag.hex()] for t in r["terms"]],
        })
    out["circuits"] = circuits
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", os.path.join(HERE, "golden.json"))


if __name__ == "__main__":
    main()
