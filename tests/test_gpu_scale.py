"""FP64 parity at the benchmark's own large sizes, through the default whole-grid path (GPU).

The oracle results in tests/golden/scale.npz (written by tests/golden/make_scale.py on a CPU
box) are for (H2O)500 (1500 atoms, 3000 AOs), C200H402 (602 atoms, 1202 AOs) and (H2O)1000
(3000 atoms, 6000 AOs) at SCF accuracy 1e-3. Every one of these has at least 1024 AOs, so its
dense algebra runs on the whole cooperative grid (no threshold override). Bars as for the small
molecules: |dE| <= 1e-9 Eh, max|dG| <= 1e-8 Eh/bohr, charges to 1e-7 e.
"""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIX = Path(__file__).resolve().parent / "golden" / "scale.npz"
E_TOL, G_TOL = 1e-9, 1e-8


def _case(name):
    import sys

    sys.path.insert(0, str(FIX.parent))
    from make_scale import cases, checksum

    z, x = cases()[name]
    ref = np.load(FIX)
    assert len(z) == int(ref[f"{name}_natoms"])
    assert abs(checksum(x) - float(ref[f"{name}_xsum"])) <= 1e-9 * abs(float(ref[f"{name}_xsum"]))
    return z, x, ref


@pytest.mark.parametrize("name", ["c200", "w500", "w1000"])
def test_large_molecule_matches_oracle(engine, name):
    z, x, ref = _case(name)
    acc = float(ref["accuracy"])
    nao = engine.basis_size(z)[1]
    assert nao >= 1024  # the whole-grid path
    r = engine.Calculator(z, x, accuracy=acc).singlepoint(x, levels=False)
    assert r.status == 0 and r.converged
    de = abs(r.energy - float(ref[f"{name}_energy"]))
    dg = float(np.abs(r.gradient - ref[f"{name}_gradient"]).max())
    dq = float(np.abs(r.charges - ref[f"{name}_qat"]).max())
    names = ("repulsion", "dispersion", "electronic", "isotropic_es", "third_order", "anisotropic", "entropy", "band")
    dterms = {k: float(r.terms[k] - t) for k, t in zip(names, ref[f"{name}_terms"])}
    print(f"{name}: {len(z)} atoms, {nao} AOs, |dE| = {de:.2e} Eh, max|dG| = {dg:.2e} Eh/bohr, max|dq| = {dq:.2e}, "
          f"{r.iterations} iterations (oracle {int(ref[f'{name}_iterations'])}); term differences {dterms}")
    assert de < E_TOL
    assert dg < G_TOL
    assert dq < 1e-7
