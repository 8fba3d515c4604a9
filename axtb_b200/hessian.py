"""Semi-numerical Hessian from central differences of analytic gradients, the displacements in
batches on the GPU.

axtb's numerical Hessian (``Calculator::numerical_hessian``, crates/axtb/src/calculator.rs:266-296,
with crates/base/src/fd.rs:39-41, 122-140, 170-207): one reference single point, then every
Cartesian coordinate moved forward by the step and back by twice the step, every displaced SCF
converged to min(accuracy, 0.01) starting from the reference's converged moments (a displaced
SCF that does not converge from them is an error, with no second run from the guess); row y of
the matrix holds the central difference of the gradients along coordinate y (its column y, the
same once symmetrized), the matrix is replaced by its symmetric part (the largest asymmetry is
reported), and the dipole derivatives come from the same points. Here the reference is one
single point and the 6N displaced single points run as ``Batch`` runs of as many copies as fit
the free device memory, each copy seeded with the reference's moments.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .calculator import AxtbError, Batch, SinglePoint, basis_size

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


def copies_that_fit(nao: int, ncopies: int, device: int = 0) -> int:
    """How many copies of an nao-AO molecule one batch may hold: the engine keeps about 23 dense
    nao x nao FP64 planes per molecule, and a batch gets at most half of the free device memory."""
    per = 8.0 * 23.0 * max(nao, 64) ** 2 + 1.0e6
    try:
        import torch

        free = torch.cuda.mem_get_info(device)[0]
    except Exception:
        free = 16.0e9
    return max(1, min(ncopies, int(0.5 * free / per)))


def numerical_hessian(numbers, positions, charge=0.0, uhf=None, step=0.005, accuracy=None, max_batch=None,
                      **options) -> Hessian:
    """Semi-numerical Hessian of one molecule (positions in bohr; step in bohr, 0.005 axtb's
    suggestion). ``accuracy``: the SCF accuracy of the reference and displaced points (default
    0.01, never looser than the options' own accuracy); ``max_batch``: most displaced copies per
    batch (default: as many as fit half of the free device memory); the other options as for
    ``Calculator``."""
    if not (step > 0.0 and np.isfinite(step)):
        raise AxtbError(1, f"the Hessian step must be a positive number, got {step}")
    x0 = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    acc = min(NUMERICAL_ACCURACY if accuracy is None else float(accuracy), float(options.pop("accuracy", 1.0)))
    z = np.asarray(numbers, dtype=np.int32)
    # the reference single point, once; its converged moments start every displaced SCF
    ref = Batch([(z, x0, charge, uhf)], accuracy=acc, **options)
    try:
        first = ref.run(gradient=True)[0]
        if first.status != 0:
            raise AxtbError(first.status, "the reference single point of the Hessian failed")
        start = ref.get_moments(0)
    finally:
        ref.close()
    pts = displacements(x0, step)
    chunk = int(max_batch) if max_batch else copies_that_fit(basis_size(z)[1], len(pts), options.get("device", 0))
    res = []
    for c0 in range(0, len(pts), chunk):
        part = pts[c0:c0 + chunk]
        batch = Batch([(z, p, charge, uhf) for p in part], accuracy=acc, **options)
        try:
            batch.set_restart(True, retry_fresh=False)
            for i in range(len(part)):
                batch.set_moments(i, start)
            res += batch.run(gradient=True)
        finally:
            batch.close()
    bad = [i for i, r in enumerate(res) if r.status != 0]
    if bad:
        raise AxtbError(res[bad[0]].status, f"{len(bad)} displaced single points of the Hessian failed")
    gp = [r.gradient for r in res[0::2]]
    gm = [r.gradient for r in res[1::2]]
    dp = [r.dipole for r in res[0::2]]
    dm = [r.dipole for r in res[1::2]]
    h, dipd, asym = assemble(gp, gm, dp, dm, step)
    return Hessian(hessian=h, dipole_derivatives=dipd, max_asymmetry=asym, reference=first)
