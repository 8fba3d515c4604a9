"""The seeded synthetic workloads follow the benchmark configurations' geometric rules (CPU).

Water clusters: rigid waters (O-H 0.96 A, H-O-H 104.5 deg) with oxygens on a 3.1 A cubic lattice
jittered by at most 0.2 A per axis; alkanes: C-C 1.53 A, C-H 1.09 A, tetrahedral angles, a given
gauche fraction; the mixed batch: half water clusters n ~ U{5..100}, half alkanes k ~ U{5..60}."""
import numpy as np
import pytest

from axtb_b200 import structures as S

A = 1.0 / S.AATOAU  # bohr -> Angstrom


def _angle(a, b, c):
    u, v = a - b, c - b
    return np.degrees(np.arccos(np.dot(u, v) / np.linalg.norm(u) / np.linalg.norm(v)))


@pytest.mark.parametrize("n,dims", [(32, (4, 4, 2)), (500, (10, 10, 5)), (1000, (10, 10, 10))])
def test_water_cluster_rules(n, dims):
    z, x = S.water_cluster(n, seed=0, dims=dims)
    assert len(z) == 3 * n and list(z[:3]) == [8, 1, 1]
    xa = x * A
    for w in range(n):
        o, h1, h2 = xa[3 * w], xa[3 * w + 1], xa[3 * w + 2]
        assert abs(np.linalg.norm(h1 - o) - 0.96) < 1e-9 and abs(np.linalg.norm(h2 - o) - 0.96) < 1e-9
        assert abs(_angle(h1, o, h2) - 104.5) < 1e-7
    # oxygens: lattice site (filled in x, y, z order) + jitter of at most 0.2 A per axis
    a, b, c = dims
    sites = np.array([(i, j, k) for k in range(c) for j in range(b) for i in range(a)][:n], dtype=float) * 3.1
    off = xa[0::3] - sites
    assert np.abs(off).max() <= 0.2 + 1e-12
    assert np.abs(off).max() > 0.15  # the jitter is there


def test_water_box_is_near_cubic():
    for n in (5, 17, 64, 100):
        a, b, c = S._box(n)
        assert a * b * c >= n and a - c <= 1 and a >= b >= c


def test_alkane_rules():
    k = 200
    z, x = S.alkane(k, seed=3, gauche=0.1)
    assert (z == 6).sum() == k and (z == 1).sum() == 2 * k + 2
    xa = x * A
    c = xa[z == 6]
    h = xa[z == 1]
    cc = np.linalg.norm(np.diff(c, axis=0), axis=1)
    assert np.allclose(cc, 1.53, atol=1e-9)
    for i in range(1, k - 1):
        assert abs(_angle(c[i - 1], c[i], c[i + 1]) - np.degrees(S.TETRA)) < 1e-6
    # every hydrogen 1.09 A from its nearest carbon
    dch = np.linalg.norm(h[:, None] - c[None], axis=-1).min(axis=1)
    assert np.allclose(dch, 1.09, atol=1e-9)
    # dihedrals: anti (180) or gauche (+-60), about a tenth gauche
    dih = []
    for i in range(k - 3):
        b0, b1, b2 = c[i + 1] - c[i], c[i + 2] - c[i + 1], c[i + 3] - c[i + 2]
        n1, n2 = np.cross(b0, b1), np.cross(b1, b2)
        m = np.cross(n1, b1 / np.linalg.norm(b1))
        dih.append(np.degrees(np.arctan2(np.dot(m, n2), np.dot(n1, n2))))
    dih = np.abs(np.array(dih))
    gauche = np.isclose(dih, 60.0, atol=1e-6)
    assert np.all(gauche | np.isclose(dih, 180.0, atol=1e-6))
    assert 5 <= gauche.sum() <= 40


def test_generators_are_seeded():
    z1, x1 = S.alkane(30, seed=7, gauche=0.3)
    z2, x2 = S.alkane(30, seed=7, gauche=0.3)
    assert np.array_equal(z1, z2) and np.array_equal(x1, x2)
    assert not np.array_equal(S.water_cluster(20, seed=1)[1], S.water_cluster(20, seed=2)[1])


def test_mixed_batch_composition():
    mols = S.mixed_batch(256, seed=0)
    waters = [z for z, _ in mols if not (z == 6).any()]
    alkanes = [z for z, _ in mols if (z == 6).any()]
    assert len(waters) == len(alkanes) == 128
    nw = np.array([len(z) // 3 for z in waters])
    kc = np.array([(z == 6).sum() for z in alkanes])
    assert nw.min() >= 5 and nw.max() <= 100 and kc.min() >= 5 and kc.max() <= 60
    assert np.ptp(nw) > 60 and np.ptp(kc) > 35  # spread over the ranges
