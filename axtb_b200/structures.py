"""Seeded synthetic molecules of the benchmark workloads (positions in bohr).

* ``water_cluster(n, seed)``: n rigid waters (O-H 0.96 A, H-O-H 104.5 deg) on a cubic lattice of
  3.1 A spacing (the smallest near-cubic box holding n sites, filled in order), each oxygen
  jittered by U(-0.2, 0.2) A per axis and each molecule rotated uniformly at random.
* ``alkane(k, seed, gauche)``: C_kH_(2k+2) zigzag chain, C-C 1.53 A, C-H 1.09 A, tetrahedral
  angles, each C-C-C-C dihedral gauche (+-60 deg) with probability ``gauche`` else anti.
* ``mixed_batch``, ``adjoint_batch``: the batched workloads built from these rules.

Angstrom to bohr with the CODATA 2022 Bohr radius (crates/base/src/units.rs:18-21).
"""
from __future__ import annotations

import numpy as np

AATOAU = 1.0 / 0.529177210544
TETRA = np.arccos(-1.0 / 3.0)  # 109.47 deg


def _rotation(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _box(n: int):
    """Smallest near-cubic box (a >= b >= c, a - c <= 1) holding n sites."""
    best = None
    for c in range(1, n + 1):
        for b in (c, c + 1):
            for a in (b, b + 1):
                if a - c > 1 or a * b * c < n:
                    continue
                if best is None or a * b * c < best[0] * best[1] * best[2]:
                    best = (a, b, c)
        if c * c * c > n:
            break
    return best


def water_cluster(n: int, seed: int = 0, dims=None, spacing: float = 3.1, jitter: float = 0.2):
    rng = np.random.default_rng(seed)
    a, b, c = dims if dims is not None else _box(n)
    sites = [(i, j, k) for k in range(c) for j in range(b) for i in range(a)][:n]
    roh, ang = 0.96, np.deg2rad(104.5)
    mono = np.array([[0.0, 0.0, 0.0],
                     [roh * np.sin(ang / 2), 0.0, roh * np.cos(ang / 2)],
                     [-roh * np.sin(ang / 2), 0.0, roh * np.cos(ang / 2)]])
    numbers, pos = [], []
    for s in sites:
        o = np.array(s, dtype=float) * spacing + rng.uniform(-jitter, jitter, 3)
        r = _rotation(rng)
        for z, v in zip((8, 1, 1), mono):
            numbers.append(z)
            pos.append(o + r @ v)
    return np.array(numbers, dtype=np.int32), np.array(pos) * AATOAU


def _place(a, b, c, bond, angle, dihedral):
    """Position of D with |CD| = bond, angle BCD, dihedral ABCD (natural extension reference frame)."""
    bc = c - b
    bc /= np.linalg.norm(bc)
    nrm = np.cross(b - a, bc)
    nrm /= np.linalg.norm(nrm)
    m = np.array([bc, np.cross(nrm, bc), nrm]).T
    d2 = bond * np.array([-np.cos(angle), np.sin(angle) * np.cos(dihedral), np.sin(angle) * np.sin(dihedral)])
    return c + m @ d2


def _clash_free(numbers, pos) -> bool:
    """No contact shorter than the covalent geometry's own 1-3 distances (H-H 1.7 A, C-H 2.0 A
    unless bonded, C-C 2.4 A unless bonded)."""
    d = np.linalg.norm(pos[:, None] - pos[None], axis=-1) / AATOAU
    iu = np.triu_indices(len(numbers), 1)
    zz = numbers[iu[0]] + numbers[iu[1]]
    dd = d[iu]
    hh = dd[zz == 2].min(initial=9.0) >= 1.7
    ch = ((dd[zz == 7] < 1.2) | (dd[zz == 7] >= 2.0)).all()
    cc = ((dd[zz == 12] < 1.6) | (dd[zz == 12] >= 2.4)).all()
    return bool(hh and ch and cc)


def alkane(k: int, seed: int = 0, gauche: float = 0.3):
    """Chains whose random dihedrals fold back onto themselves are drawn again from the next
    seed (deterministically); a gauche following a gauche keeps its sign (g+g- is the
    sterically forbidden syn-pentane contact)."""
    for attempt in range(1000):
        z, x = _alkane_draw(k, seed + 7777 * attempt, gauche)
        if _clash_free(z, x):
            return z, x
    raise RuntimeError("no clash-free alkane conformer")


def _alkane_draw(k: int, seed: int, gauche: float):
    rng = np.random.default_rng(seed)
    rcc, rch = 1.53, 1.09
    cs = [np.array([0.0, 0.0, 0.0]), np.array([rcc, 0.0, 0.0])]
    if k >= 3:
        cs.append(cs[1] + rcc * np.array([-np.cos(TETRA), np.sin(TETRA), 0.0]))
    prev = np.pi
    for i in range(3, k):
        dih = np.pi
        if rng.random() < gauche:
            sgn = (1 if rng.random() < 0.5 else -1) if prev == np.pi else np.sign(prev)
            dih = np.deg2rad(60.0) * sgn
        prev = dih
        cs.append(_place(cs[i - 3], cs[i - 2], cs[i - 1], rcc, TETRA, dih))
    cs = cs[:k]
    hs = []
    for i in range(k):
        if 0 < i < k - 1:
            # two hydrogens: +-120 deg dihedral from the chain continuation
            for sgn in (1, -1):
                hs.append(_place(cs[i + 1], cs[i - 1], cs[i], rch, TETRA, sgn * 2 * np.pi / 3))
        else:
            nb = cs[1] if i == 0 else cs[k - 2]
            nb2 = cs[2] if i == 0 and k > 2 else (cs[k - 3] if k > 2 else nb + np.array([0.0, 1.0, 0.0]))
            for dih in (np.pi, np.pi / 3, -np.pi / 3):
                hs.append(_place(nb2, nb, cs[i], rch, TETRA, dih))
    numbers = np.array([6] * k + [1] * len(hs), dtype=np.int32)
    return numbers, np.array(cs + hs) * AATOAU


def mixed_batch(nmol: int = 4096, seed: int = 0):
    """Half water clusters (H2O)n with n ~ U{5..100}, half alkanes C_kH_(2k+2) with k ~ U{5..60}
    (dihedrals anti 70 % / gauche 30 %)."""
    rng = np.random.default_rng(seed)
    mols = []
    for i in range(nmol):
        if i % 2 == 0:
            mols.append(water_cluster(int(rng.integers(5, 101)), seed=seed * 100003 + i))
        else:
            mols.append(alkane(int(rng.integers(5, 61)), seed=seed * 100003 + i, gauche=0.3))
    return mols


def adjoint_batch(nmol: int = 512, seed: int = 0, noise: float = 0.05):
    """Alkanes (k ~ U{10..40}) and water clusters (n ~ U{10..60}), each with N(0, noise A)
    coordinate noise."""
    rng = np.random.default_rng(seed)
    mols = []
    for i in range(nmol):
        if i < nmol // 2:
            z, x = alkane(int(rng.integers(10, 41)), seed=seed * 7919 + i, gauche=0.3)
        else:
            z, x = water_cluster(int(rng.integers(10, 61)), seed=seed * 7919 + i)
        mols.append((z, x + rng.normal(0.0, noise * AATOAU, x.shape)))
    return mols
