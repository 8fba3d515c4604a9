"""Semi-numerical Hessian from central differences of analytic gradients, all displacements in
one batch on the GPU.

axtb's numerical Hessian (``Calculator::numerical_hessian``, crates/axtb/src/calculator.rs:266-296,
with crates/base/src/fd.rs:39-41, 122-140, 170-207): a reference single point, then every
Cartesian coordinate moved forward by the step and back by twice the step, every displaced SCF
converged to min(accuracy, 0.01) starting from the reference's converged moments; row y of the
matrix holds the central difference of the gradients along coordinate y (its column y, the same
once symmetrized), the matrix is replaced by its symmetric part (the largest asymmetry is
reported), and the dipole derivatives come from the same points. Here the 6N displaced single
points are one ``Batch`` run, each molecule restarting from the reference's moments.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .calculator import AxtbError, Batch, SinglePoint

NUMERICAL_ACCURACY = 0.01  # crates/axtb/src/calculator.rs:86


@dataclass
class Hessian:
    hessian: np.ndarray              # (3N, 3N), Eh/bohr^2, symmetric
    dipole_derivatives: np.ndarray   # (3N, 3), d mu / d x_y (e)
    max_asymmetry: float             # largest |H_ij - H_ji| before symmetrizing
    reference: SinglePoint           # the single point at the reference geometry


def displacements(positions: np.ndarray, step: float) -> list[np.ndarray]:
    """The 6N displaced geometries, coordinate by coordinate: forward by the step, then back by
    twice the step from there (fd.rs:180-190, Displacement::ForwardBack)."""
    x0 = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    out = []
    for y in range(x0.size):
        a, k = divmod(y, 3)
        xp = x0.copy()
        xp[a, k] = x0[a, k] + step
        xm = xp.copy()
        xm[a, k] = xp[a, k] - 2.0 * step
        out += [xp, xm]
    return out


def assemble(gplus, gminus, dplus, dminus, step: float):
    """Central differences (p - m) / (2 step) of the gradients (row y = coordinate y) and dipoles,
    then the symmetric part of the matrix; returns (hessian, dipole derivatives, max asymmetry)."""
    gp = np.asarray(gplus, dtype=np.float64).reshape(len(gplus), -1)
    gm = np.asarray(gminus, dtype=np.float64).reshape(len(gminus), -1)
    h = (gp - gm) / (2.0 * step)
    n = h.shape[0]
    if h.shape != (n, n):
        raise ValueError(f"{n} displaced gradients of {h.shape[1]} entries")
    asym = float(np.abs(h - h.T).max()) if n else 0.0
    upper = np.triu_indices(n, 1)
    sym = 0.5 * (h[upper[1], upper[0]] + h[upper])
    h[upper] = sym
    h[upper[1], upper[0]] = sym
    dipd = (np.asarray(dplus, dtype=np.float64) - np.asarray(dminus, dtype=np.float64)) / (2.0 * step)
    return h, dipd, asym


def numerical_hessian(numbers, positions, charge=0.0, uhf=None, step=0.005, accuracy=None, **options) -> Hessian:
    """Semi-numerical Hessian of one molecule (positions in bohr; step in bohr, 0.005 axtb's
    suggestion). ``accuracy``: the SCF accuracy of the displaced points (default 0.01, never
    looser than the options' own accuracy); the other options as for ``Calculator``."""
    if not (step > 0.0 and np.isfinite(step)):
        raise AxtbError(1, f"the Hessian step must be a positive number, got {step}")
    x0 = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    acc = min(NUMERICAL_ACCURACY if accuracy is None else float(accuracy), float(options.pop("accuracy", 1.0)))
    pts = displacements(x0, step)
    z = np.asarray(numbers, dtype=np.int32)
    batch = Batch([(z, x0, charge, uhf)] * (1 + len(pts)), accuracy=acc, **options)
    try:
        batch.set_restart(True)
        first = batch.run(gradient=True)  # the reference single point (every copy holds its moments)
        if first[0].status != 0:
            raise AxtbError(first[0].status, "the reference single point of the Hessian failed")
        res = batch.run(positions=[x0] + pts, gradient=True)
        bad = [i for i, r in enumerate(res[1:]) if r.status != 0]
        if bad:
            raise AxtbError(res[1 + bad[0]].status, f"{len(bad)} displaced single points of the Hessian failed")
        gp = [r.gradient for r in res[1::2]]
        gm = [r.gradient for r in res[2::2]]
        dp = [r.dipole for r in res[1::2]]
        dm = [r.dipole for r in res[2::2]]
        h, dipd, asym = assemble(gp, gm, dp, dm, step)
        return Hessian(hessian=h, dipole_derivatives=dipd, max_asymmetry=asym, reference=first[0])
    finally:
        batch.close()
