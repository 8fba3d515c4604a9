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


def test_moments_seed_another_calculator(engine):
    """Session lineages across calculators (Method::wavefunction / set_wavefunction /
    set_history, crates/axtb/src/calculator.rs:413-447, through axtb_gpu_get_moments and
    axtb_gpu_set_moments): a fresh calculator seeded with another's converged moments takes the
    same warm-started SCF as that calculator itself (same iterations, same bits), and a batch
    molecule seeded the same way through axtb_gpu_batch_set_moments agrees with it."""
    from axtb_b200 import structures as S

    z, x = S.water_cluster(12, seed=7)
    moved = x + np.random.default_rng(1).normal(scale=0.02, size=x.shape)
    a = engine.Calculator(z, x, accuracy=1e-6)
    assert a.wavefunction() is None
    a.singlepoint(x)
    w = a.wavefunction()
    assert w is not None and w.qsh.size == engine.basis_size(z)[0]
    ra = a.singlepoint(moved)  # warm start from its own moments at x
    cold = engine.Calculator(z, x, accuracy=1e-6).singlepoint(moved)
    assert ra.iterations < cold.iterations
    for given in (True, False):
        b = engine.Calculator(z, x, accuracy=1e-6)
        (b.set_wavefunction if given else b.set_history)(w)
        rb = b.singlepoint(moved)
        assert rb.iterations == ra.iterations
        assert rb.energy == ra.energy and np.array_equal(rb.gradient, ra.gradient)
    c = engine.Calculator(z, x, accuracy=1e-6)
    c.set_history(w)
    c.set_history(None)  # forgotten: a cold start
    assert c.singlepoint(moved).iterations == cold.iterations
    batch = engine.Batch([(z, moved)], accuracy=1e-6)
    batch.set_moments(0, w)
    rbt = batch.run()[0]
    assert rbt.iterations == ra.iterations and abs(rbt.energy - ra.energy) < 1e-12
    wb = batch.get_moments(0)
    assert np.abs(wb.qsh - rb.qsh).max() < 1e-10
    batch.close()


def test_dispersion_off_matches_oracle(engine, golden):
    """Options::dispersion = false (crates/axtb/src/lib.rs:185-187) leaves the D4 term out; the
    oracle with the same switch gives the same energy and gradient, and the dispersion term is 0."""
    from oracle import oracle as O

    c = golden["struct-caffeine"]
    z, x = np.array(c["numbers"]), np.array(c["positions"])
    r = engine.Calculator(z, x, accuracy=1e-6, dispersion=False).singlepoint(x)
    ref = O.singlepoint(z, x, accuracy=1e-6, dispersion=False)
    full = O.singlepoint(z, x, accuracy=1e-6)
    assert r.terms["dispersion"] == 0.0 and ref["terms"]["dispersion"] == 0.0
    assert abs(full["energy"] - ref["energy"]) > 1e-3
    assert abs(r.energy - ref["energy"]) < 1e-9
    assert np.abs(r.gradient - ref["gradient"]).max() < 1e-8
