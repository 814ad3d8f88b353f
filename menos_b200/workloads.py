"""Seeded synthetic workloads of the dense statevector path.

No public benchmark suite stands behind these; they are the circuit families
the engine is measured on, generated from a fixed seeding convention:
  * angles come from std::mt19937_64(seed), each uniform as the reference's
    common::Rng maps a word, (w >> 11) * 2^-53 (src/common/rng.cpp:184-186),
    scaled to the stated interval;
  * a Pauli string takes one word per qubit, w % 4 -> I / X / Y / Z;
  * weights are N(0, 1) by Box-Muller from the same stream.

Families:
  brick(n, depth, seed)       U3(theta, phi, lambda in [0, 2pi)) on every qubit, then CZ on
                              (0,1),(2,3),... on even layers, (1,2),(3,4),... on odd layers
  qft(n)                      H(j), CP(2pi / 2^(k-j+1)) on (k, j) for k > j, then the final swaps
  hea(n, layers, seed)        RY(theta) RZ(phi) on every qubit (angles in [-pi, pi)) + CX(q, q+1) ladder
  pauli_strings(n, count, seed), weights(count, seed)
"""
from __future__ import annotations

import math

from .circuit import Circuit

_MASK64 = (1 << 64) - 1


class MT19937_64:
    """The 64-bit Mersenne Twister (Matsumoto & Nishimura), with the
    parameters the C++ standard fixes for std::mt19937_64."""

    def __init__(self, seed: int):
        mt = [0] * 312
        mt[0] = seed & _MASK64
        for i in range(1, 312):
            mt[i] = (6364136223846793005 * (mt[i - 1] ^ (mt[i - 1] >> 62)) + i) & _MASK64
        self.mt = mt
        self.idx = 312

    def _twist(self):
        mt = self.mt
        for i in range(312):
            y = (mt[i] & 0xFFFFFFFF80000000) | (mt[(i + 1) % 312] & 0x7FFFFFFF)
            v = mt[(i + 156) % 312] ^ (y >> 1)
            if y & 1:
                v ^= 0xB5026F5AA96619E9
            mt[i] = v
        self.idx = 0

    def next_word(self) -> int:
        if self.idx >= 312:
            self._twist()
        x = self.mt[self.idx]
        self.idx += 1
        x ^= (x >> 29) & 0x5555555555555555
        x ^= (x << 17) & 0x71D67FFFEDA60000
        x ^= (x << 37) & 0xFFF7EEE000000000
        x ^= x >> 43
        return x & _MASK64

    def uniform(self) -> float:
        """(w >> 11) * 2^-53, exactly as common::Rng::word_to_uniform."""
        return float(self.next_word() >> 11) * (1.0 / 9007199254740992.0)


TWO_PI = 2.0 * math.pi


def brick(n: int, depth: int, seed: int, circ: Circuit | None = None) -> Circuit:
    c = circ if circ is not None else Circuit(n)
    rng = MT19937_64(seed)
    for layer in range(depth):
        for q in range(n):
            theta = TWO_PI * rng.uniform()
            phi = TWO_PI * rng.uniform()
            lam = TWO_PI * rng.uniform()
            c.gate("u", [q], [theta, phi, lam])
        start = 0 if layer % 2 == 0 else 1
        for q in range(start, n - 1, 2):
            c.gate("cz", [q, q + 1])
    return c


def qft(n: int, circ: Circuit | None = None) -> Circuit:
    c = circ if circ is not None else Circuit(n)
    for j in range(n):
        c.gate("h", [j])
        for k in range(j + 1, n):
            c.gate("cp", [k, j], [TWO_PI / float(1 << (k - j + 1))])
    for i in range(n // 2):
        c.gate("swap", [i, n - 1 - i])
    return c


def hea(n: int, layers: int, seed: int, circ: Circuit | None = None) -> Circuit:
    c = circ if circ is not None else Circuit(n)
    rng = MT19937_64(seed)
    for _ in range(layers):
        for q in range(n):
            theta = -math.pi + TWO_PI * rng.uniform()
            phi = -math.pi + TWO_PI * rng.uniform()
            c.gate("ry", [q], [theta])
            c.gate("rz", [q], [phi])
        for q in range(n - 1):
            c.gate("cx", [q, q + 1])
    return c


CROSSOVER_LAYERS = 6


def crossover(n: int, circ: Circuit | None = None) -> Circuit:
    """The chunked tier's crossover family (benchmarks/crossover_circuit.h:
    make_crossover_circuit): per layer H on every qubit, T on qubit 0, then
    CX on neighbour pairs starting at qubit layer % 2; six layers."""
    c = circ if circ is not None else Circuit(n)
    for layer in range(CROSSOVER_LAYERS):
        for q in range(n):
            c.gate("h", [q])
        c.gate("t", [0])
        for q in range(layer % 2, n - 1, 2):
            c.gate("cx", [q, q + 1])
    return c


def ladder(n: int, circ: Circuit | None = None) -> Circuit:
    """The chunked tier's ladder family (tests/engines/dense_tiered/
    pass_plan_test.cpp: ladder): per layer H on every qubit, then the CX
    chain q -> q + 1; six layers."""
    c = circ if circ is not None else Circuit(n)
    for _ in range(CROSSOVER_LAYERS):
        for q in range(n):
            c.gate("h", [q])
        for q in range(n - 1):
            c.gate("cx", [q, q + 1])
    return c


def hea_bindings(n: int, layers: int, count: int, seed: int):
    """`count` parameter rows for hea(n, layers): per layer and qubit RY(theta)
    then RZ(phi), angles in [-pi, pi) from mt19937_64(seed), in op order."""
    rng = MT19937_64(seed)
    return [[-math.pi + TWO_PI * rng.uniform() for _ in range(2 * n * layers)] for _ in range(count)]


def pauli_strings(n: int, count: int, seed: int):
    """(x_mask, z_mask) pairs; per qubit w % 4 -> I, X, Y, Z."""
    rng = MT19937_64(seed)
    out = []
    for _ in range(count):
        x = z = 0
        for q in range(n):
            r = rng.next_word() % 4
            if r == 1:
                x |= 1 << q
            elif r == 2:
                x |= 1 << q
                z |= 1 << q
            elif r == 3:
                z |= 1 << q
        out.append((x, z))
    return out


def weights(count: int, seed: int):
    """N(0,1) by Box-Muller on (1 - u1, u2)."""
    rng = MT19937_64(seed)
    out = []
    for _ in range(count):
        u1 = 1.0 - rng.uniform()
        u2 = rng.uniform()
        out.append(math.sqrt(-2.0 * math.log(u1)) * math.cos(TWO_PI * u2))
    return out


def config_c1(seed: int = 20260929) -> Circuit:
    """20 qubits, 20 brick layers (statevector + 4096 shots)."""
    return brick(20, 20, seed)


def config_c2(n: int = 30, depth: int = 40, seed: int = 20260929) -> Circuit:
    """The 30-qubit complex128 workload: brick depth 40, then a full QFT."""
    c = brick(n, depth, seed)
    return qft(n, c)


def serving_stream(count: int, rate: float, seed: int, nmin: int = 12, nmax: int = 28, dmin: int = 4,
                   dmax: int = 40, shots: int = 4096, terms: int = 32):
    """Requests of the serving workload: Poisson arrivals at `rate` per
    second; qubits uniform in [nmin, nmax], depth uniform in [dmin, dmax]
    layers of the U3/CZ brick or the RY/RZ + CX ansatz; each asks for
    `shots` counts or <H> over `terms` weighted Pauli strings.  Returns a
    list of dicts (arrival_s, circuit, output, shots, seed, paulis, coefs)."""
    rng = MT19937_64(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += -math.log(1.0 - rng.uniform()) / rate
        n = nmin + int(rng.uniform() * (nmax - nmin + 1))
        depth = dmin + int(rng.uniform() * (dmax - dmin + 1))
        family = "brick" if rng.uniform() < 0.5 else "hea"
        cseed = rng.next_word()
        circ = brick(n, depth, cseed) if family == "brick" else hea(n, depth, cseed)
        if rng.uniform() < 0.5:
            out.append({"arrival_s": t, "circuit": circ, "output": "counts", "shots": shots,
                        "seed": rng.next_word(), "paulis": (), "coefs": (), "family": family})
        else:
            ps = pauli_strings(n, terms, rng.next_word())
            ws = weights(terms, rng.next_word())
            out.append({"arrival_s": t, "circuit": circ, "output": "expectation", "shots": 0, "seed": 0,
                        "paulis": ps, "coefs": ws, "family": family})
    return out
