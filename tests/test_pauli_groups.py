"""Grouping of Pauli terms for the expectation reduction, checked on the CPU:
the plan mb2_expectation runs (mb2_debug_pauli_groups) is emulated in numpy
and must visit every amplitude pair (m, m ^ x) of every term exactly once,
tile by tile, and reproduce <psi|P|psi> of the oracle's formula
(src/kernels/cpu/dense_kernels.cpp:544-569)."""
import ctypes as C

import numpy as np
import pytest

from menos_b200 import _lib


def plan(terms, n):
    xs = np.ascontiguousarray([t[0] for t in terms], np.uint64)
    zs = np.ascontiguousarray([t[1] for t in terms], np.uint64)
    words = C.c_uint64(0)
    L = _lib.lib()
    assert L.mb2_debug_pauli_groups(xs.ctypes.data, zs.ctypes.data, len(terms), n, None, C.byref(words)) == 1
    out = np.zeros(words.value, np.uint64)
    assert L.mb2_debug_pauli_groups(xs.ctypes.data, zs.ctypes.data, len(terms), n, out.ctypes.data,
                                    C.byref(words)) == 0
    w = [int(v) for v in out]
    groups, i = [], 1
    for _ in range(w[0]):
        c, d, free, nt = w[i:i + 4]
        i += 4
        span = w[i:i + (1 << d)]
        i += 1 << d
        ts = []
        for _ in range(nt):
            ts.append(tuple(w[i:i + 3]))
            i += 3
        groups.append((c, d, free, span, ts))
    assert i == len(w)
    return groups


def deposit(v, mask):
    r, b = 0, 0
    while mask:
        low = mask & -mask
        if (v >> b) & 1:
            r |= low
        b += 1
        mask ^= low
    return r


def tiles_of(c, d, free, span, n):
    ncos = 1 << bin(free).count("1")
    assert ncos == 1 << (n - c - d)
    for cs in range(ncos):
        rep = deposit(cs, free)
        yield [((rep ^ span[L >> c]) << c) | (L & ((1 << c) - 1)) for L in range(1 << (c + d))]


def emulate(groups, terms, psi, n):
    out = np.zeros(len(terms), np.complex128)
    seen_terms = []
    for c, d, free, span, ts in groups:
        assert c + d <= 12 and d <= 9 and 1 <= len(ts) <= 16
        covered = np.zeros(1 << n, np.int64)
        pairs = {t[0]: set() for t in ts}
        for tile in tiles_of(c, d, free, span, n):
            covered[tile] += 1
            for idx, kx, xl in ts:
                x, z = terms[idx]
                dl = (kx << c) | xl
                for L in range(len(tile)):
                    if dl and (L >> (dl.bit_length() - 1)) & 1:
                        continue
                    m, m2 = tile[L], tile[L ^ dl]
                    assert m2 == m ^ x
                    key = (min(m, m2), max(m, m2))
                    assert key not in pairs[idx]
                    pairs[idx].add(key)
                    a, b = psi[m], psi[m2]
                    s1 = -1 if bin(z & m).count("1") & 1 else 1
                    if dl == 0:
                        out[idx] += s1 * abs(a) ** 2
                    else:
                        s2 = -1 if bin(z & m2).count("1") & 1 else 1
                        t = np.conj(a) * b
                        out[idx] += s2 * t + s1 * np.conj(t)
        assert (covered == 1).all()
        for idx, _, _ in ts:
            x = terms[idx][0]
            assert len(pairs[idx]) == ((1 << n) if x == 0 else (1 << (n - 1)))
            out[idx] *= 1j ** (bin(x & terms[idx][1]).count("1") & 3)
            seen_terms.append(idx)
    assert sorted(seen_terms) == list(range(len(terms)))
    return out


def direct(psi, x, z, n):
    m = np.arange(1 << n)
    par = np.array([bin(int(z) & int(v ^ x)).count("1") & 1 for v in m])
    val = np.sum(np.conj(psi) * psi[m ^ x] * np.where(par, -1.0, 1.0))
    return val * 1j ** (bin(x & z).count("1") & 3)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 9, 12, 14])
def test_groups_cover_every_pair_once(n):
    rng = np.random.default_rng(n)
    terms = [(0, 0), ((1 << n) - 1, 0), (0, (1 << n) - 1), (1, 1 << (n - 1))]
    terms += [(int(rng.integers(0, 1 << n)), int(rng.integers(0, 1 << n))) for _ in range(40)]
    terms += [(int(rng.integers(0, 8)) & ((1 << n) - 1), int(rng.integers(0, 1 << n))) for _ in range(6)]
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi /= np.linalg.norm(psi)
    got = emulate(plan(terms, n), terms, psi, n)
    for (x, z), g in zip(terms, got):
        assert abs(g - direct(psi, x, z, n)) < 1e-12


def test_random_terms_share_reads():
    # 64 random 30-qubit strings: ~9 per group (tile of 2^12), not one each.
    rng = np.random.default_rng(1)
    terms = [(int(rng.integers(0, 1 << 30)), int(rng.integers(0, 1 << 30))) for _ in range(64)]
    groups = plan(terms, 30)
    assert len(groups) <= 9
    assert sum(len(g[4]) for g in groups) == 64
    # Z strings and low-X strings join an existing group without growing it.
    zs = [(0, int(rng.integers(0, 1 << 30))) for _ in range(10)] + [(5, 3)]
    assert len(plan(zs, 30)) == 1
