"""Semi-numerical Hessian on the GPU (axtb_b200.hessian; GPU).

The 18 displaced single points of water in one batch, restarting from the reference's moments:
the matrix equals the same central differences of the oracle's gradients (1e-6 Eh/bohr^2, SCF
accuracy 1e-8), is symmetric, and its rows sum to zero over the atoms (translations).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_numerical_hessian_matches_oracle_differences(engine, golden):
    from axtb_b200.hessian import assemble, displacements, numerical_hessian
    from oracle import oracle as O

    c = golden["struct-water"]
    z, x = np.array(c["numbers"]), np.array(c["positions"])
    step = 0.005
    hs = numerical_hessian(z, x, step=step, accuracy=1e-8)
    refs = [O.singlepoint(z, p, accuracy=1e-8) for p in displacements(x, step)]
    h, dipd, _ = assemble([r["gradient"] for r in refs[0::2]], [r["gradient"] for r in refs[1::2]],
                          [r["dipole"] for r in refs[0::2]], [r["dipole"] for r in refs[1::2]], step)
    assert np.abs(hs.hessian - h).max() < 1e-6
    assert np.abs(hs.dipole_derivatives - dipd).max() < 1e-6
    assert np.array_equal(hs.hessian, hs.hessian.T) and hs.max_asymmetry < 1e-4
    assert np.abs(hs.hessian.reshape(9, 3, 3).sum(axis=1)).max() < 1e-5
    assert abs(hs.reference.energy - O.singlepoint(z, x, accuracy=1e-8)["energy"]) < 1e-9


def test_numerical_hessian_default_accuracy_in_chunks(engine, golden):
    """At axtb's default accuracy of the displaced points (0.01) and in batches of 16 copies,
    the matrix stays within 1e-4 Eh/bohr^2 of the tightly converged one (axtb's own numerical
    Hessian differs from its analytic one by ~3e-5 at these settings) and is symmetric."""
    from axtb_b200.hessian import numerical_hessian

    c = golden["struct-caffeine"]
    z, x = np.array(c["numbers"]), np.array(c["positions"])
    tight = numerical_hessian(z, x, accuracy=1e-8)
    loose = numerical_hessian(z, x, max_batch=16)
    assert np.abs(loose.hessian - tight.hessian).max() < 1e-4
    assert np.array_equal(loose.hessian, loose.hessian.T) and loose.max_asymmetry < 1e-3
    assert abs(loose.reference.energy - tight.reference.energy) < 1e-6
