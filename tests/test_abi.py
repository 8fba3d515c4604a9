"""The C-ABI library: it builds, loads without a GPU and exports every entry point that
include/*.h declares; the host logic that needs no device (basis sizes, options) works (CPU)."""
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(?:int|void\*?|int64_t)\s+\*?(axtb_gpu_\w+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(engine):
    from axtb_b200 import _lib

    lib = _lib.load()
    names = declared()
    assert len(names) >= 14, names
    for n in names:
        assert hasattr(lib, n), n
    assert set(_lib.SIGNATURES) == names


def test_basis_sizes(engine):
    from axtb_b200 import basis_size
    from oracle import oracle as O

    for z in ([8, 1, 1], [6] * 10 + [1] * 22, [26, 6, 8, 17, 30, 1]):
        assert basis_size(z) == O.sizes(z)


def test_default_options(engine):
    from axtb_b200 import _lib

    o = _lib.default_options()
    assert (o.accuracy, o.etemp, o.max_iter, o.damping, o.guess, o.precision) == (1.0, 300.0, 250, 0.4, 0, 0)


def test_unsupported_element(engine):
    from axtb_b200 import AxtbError, basis_size

    with pytest.raises(AxtbError):
        basis_size([87, 1])


def test_structures():
    from axtb_b200 import structures as S

    z, x = S.water_cluster(32, 0, dims=(4, 4, 2))
    assert len(z) == 96 and (z == 8).sum() == 32
    d = np.linalg.norm(x[:, None] - x[None], axis=-1) + np.eye(len(z)) * 1e3
    assert abs(d.min() / S.AATOAU - 0.96) < 1e-9
    z, x = S.alkane(200, seed=3, gauche=0.1)
    assert (z == 6).sum() == 200 and (z == 1).sum() == 402
    d = np.linalg.norm(x[:, None] - x[None], axis=-1) + np.eye(len(z)) * 1e3
    assert d.min() / S.AATOAU > 1.0
    mols = S.mixed_batch(16, seed=0)
    assert len(mols) == 16
