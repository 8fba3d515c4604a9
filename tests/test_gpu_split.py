"""Split-precision mode (precision="split": the basis-transform GEMMs of F' = L^-1 F L^-T and the
energy-weighted density GEMM as BF16 tensor-core products of three-part split operands; the
eigensolver, C, P, the mixer and all sums in FP64) against the FP64 path on the same molecules
(GPU): |dE| < 1e-6 Eh, max |dG| < 1e-5 Eh/bohr."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_split_precision_error_bounds(engine):
    """At the batch workload's SCC accuracy (0.1: |dE| < 1e-7 Eh between iterations); tighter
    settings ask for energy changes below the split products' rounding floor (~1e-10 Eh) and
    are not what the mode is for."""
    from axtb_b200 import structures as S

    mols = S.mixed_batch(64, seed=5)
    ref = engine.Batch(mols, accuracy=0.1).run(gradient=True)
    spl = engine.Batch(mols, accuracy=0.1, precision="split").run(gradient=True)
    de = max(abs(a.energy - b.energy) for a, b in zip(ref, spl))
    dg = max(np.abs(a.gradient - b.gradient).max() for a, b in zip(ref, spl))
    assert all(r.status == 0 for r in spl)
    assert de < 1e-6, de
    assert dg < 1e-5, dg


def test_split_precision_option_is_validated(engine):
    with pytest.raises(KeyError):
        engine.Batch([([8, 1, 1], np.eye(3))], precision="fp16")
