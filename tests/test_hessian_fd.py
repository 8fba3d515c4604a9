"""The finite-difference layer of the semi-numerical Hessian (CPU: no engine call).

crates/base/src/fd.rs:39-41, 122-140, 170-207: coordinate y moved forward by the step and back by
twice the step; row y = the central difference of the gradients; the symmetric part with the
largest asymmetry reported; dipole derivatives from the same points.
"""
import numpy as np

from axtb_b200.hessian import assemble, displacements


def test_displacements_forward_then_back_by_twice_the_step():
    x0 = np.array([[0.1, -0.2, 0.3], [1.4, 0.0, -0.7]])
    pts = displacements(x0, 0.005)
    assert len(pts) == 12
    for y in range(6):
        a, k = divmod(y, 3)
        xp, xm = pts[2 * y], pts[2 * y + 1]
        assert xp[a, k] == x0[a, k] + 0.005 and xm[a, k] == (x0[a, k] + 0.005) - 2 * 0.005
        mask = np.ones_like(x0, dtype=bool)
        mask[a, k] = False
        assert np.array_equal(xp[mask], x0[mask]) and np.array_equal(xm[mask], x0[mask])


def test_quadratic_energy_gives_its_matrix():
    rng = np.random.default_rng(2)
    n = 9
    m = rng.normal(size=(n, n))
    a = m + m.T
    b = rng.normal(size=n)
    c = rng.normal(size=(n, 3))
    x0 = rng.normal(size=(3, 3))
    pts = displacements(x0, 0.01)
    grad = lambda x: a @ x.ravel() + b
    dip = lambda x: c.T @ x.ravel()
    h, dipd, asym = assemble([grad(p) for p in pts[0::2]], [grad(p) for p in pts[1::2]],
                             [dip(p) for p in pts[0::2]], [dip(p) for p in pts[1::2]], 0.01)
    assert np.abs(h - a).max() < 1e-10 and np.array_equal(h, h.T)
    assert asym < 1e-10
    assert np.abs(dipd - c).max() < 1e-10


def test_symmetric_part_and_asymmetry():
    g = np.array([[0.0, 2.0], [4.0, 0.0]])  # rows: gradient differences of coordinates 0 and 1
    h, _, asym = assemble([g[0] * 0.5, g[1] * 0.5], [-g[0] * 0.5, -g[1] * 0.5], [[0, 0, 0]] * 2,
                          [[0, 0, 0]] * 2, 0.5)
    assert asym == 2.0
    assert np.array_equal(h, np.array([[0.0, 3.0], [3.0, 0.0]]))
