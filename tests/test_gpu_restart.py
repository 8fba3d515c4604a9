"""Restarts across runs of a batch: each molecule starts from its previous converged moments (GPU).

axtb's calculator starts every SCF after the first from the previous geometry's converged moments
and, when that does not converge, once more from its own guess (crates/axtb/src/calculator.rs:
185-206 under Restart::Previous; the retry ladder climbs on ScfNotConverged only,
crates/base/src/method/retry.rs:119-158). ``Batch.set_restart`` does this per molecule.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_trajectory_restarts_match_cold_starts(engine):
    """A trajectory step (coordinates moved by ~0.01 bohr): starting from the previous
    moments gives the same converged energies (1e-9 Eh) and gradients (1e-8 Eh/bohr) as a cold
    start, in fewer iterations (at SCF accuracy 1e-6 the count grows with the logarithm of the
    start's error over the threshold: measured 1014 against 1159 on this batch)."""
    from axtb_b200 import structures as S

    mols = S.mixed_batch(64, seed=21)
    rng = np.random.default_rng(4)
    step = [x + rng.normal(scale=0.01, size=x.shape) for _, x in mols]
    warm = engine.Batch(mols, accuracy=1e-6)
    warm.set_restart(True)
    first = warm.run()
    assert all(r.status == 0 for r in first)
    moved = warm.run(positions=step)
    cold = engine.Batch([(z, x) for (z, _), x in zip(mols, step)], accuracy=1e-6).run()
    for rw, rc in zip(moved, cold):
        assert rw.status == rc.status == 0
        assert abs(rw.energy - rc.energy) < 1e-9
        assert np.abs(rw.gradient - rc.gradient).max() < 1e-8
    assert sum(r.iterations for r in moved) < sum(r.iterations for r in cold)
    warm.close()


def test_unconverged_restart_runs_again_from_the_guess(engine):
    """Water converged at its equilibrium geometry (SCF accuracy 10: 6 iterations), then stretched
    to 3 A with 8 iterations per attempt: the plan from the previous moments fails (8 Broyden + 8
    DIIS), so the molecule runs the plan once more from the guess, and the result is that of a
    cold start, bit for bit."""
    import json
    from pathlib import Path

    hard = json.loads((Path(__file__).parent / "golden" / "scf_hard.json").read_text())["cases"]
    c = next(h for h in hard if h["id"] == "scan-H2O-3.0-T300")
    z = np.array(c["numbers"])
    x3 = np.array(c["positions"])
    from axtb_b200 import structures as S

    zw, xw = S.water_cluster(1, seed=0, dims=(1, 1, 1))
    assert list(zw) == list(z)
    opts = dict(accuracy=10.0, max_iter=8)
    b = engine.Batch([(z, xw, 0.0, 0)], **opts)
    b.set_restart(True)
    assert b.run()[0].status == 0
    b.set_profiling(True)
    r = b.run(positions=[x3])[0]
    prof = b.profile()
    cold = engine.Batch([(z, x3, 0.0, 0)], **opts).run()[0]
    assert r.status == cold.status == 3
    assert r.iterations == cold.iterations == 16  # the fresh plan's Broyden and DIIS attempts
    assert r.energy == cold.energy and np.array_equal(r.gradient, cold.gradient)
    assert prof["kernels"]["start"]["launches"] == 2 and prof["kernels"]["start_warm"]["launches"] == 1
    b.close()
