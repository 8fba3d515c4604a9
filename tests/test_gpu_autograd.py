"""torch.autograd binding (GFN2Energy / GFN2) on the adjoint batch: 256 alkanes (k ~ U{10..40}) and
256 water clusters (n ~ U{10..60}), each with N(0, 0.05 A) coordinate noise (GPU).

backward == grad_output x the engine's analytic gradient; that gradient == the FP64 oracle's
analytic gradient on all 512 molecules (1e-8 Eh/bohr); and it matches central finite differences
(step 1e-4 bohr) along random directions on 16 sampled molecules (2e-7 Eh/bohr).
"""
import multiprocessing as mp

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ACC = 1e-6


def _oracle_gradient(mol):
    from oracle import oracle as O

    z, x = mol
    r = O.singlepoint(z, x, accuracy=ACC, lapack=True, lapack_threads=1)
    return r["energy"], r["gradient"]


@pytest.fixture(scope="module")
def adjoint():
    from axtb_b200 import structures as S

    mols = S.adjoint_batch(512, seed=0)
    # the oracle runs in spawned processes (never forked from a process that holds a GPU context)
    with mp.get_context("spawn").Pool(min(32, mp.cpu_count())) as pool:
        ref = pool.map(_oracle_gradient, mols, chunksize=4)
    return mols, ref


def _padded(mols, torch):
    nmax = max(len(z) for z, _ in mols)
    x = np.zeros((len(mols), nmax, 3))
    for i, (z, p) in enumerate(mols):
        x[i, : len(z)] = p
    return torch.tensor(x, dtype=torch.float64, device="cuda", requires_grad=True)


def test_backward_is_weighted_analytic_gradient(engine, adjoint):
    import torch

    from axtb_b200.torch_ops import GFN2

    mols, ref = adjoint
    model = GFN2(mols, accuracy=ACC)
    pos = _padded(mols, torch)
    energy = model(pos)
    w = torch.linspace(0.5, 1.5, len(mols), dtype=torch.float64, device="cuda")
    (w * energy).sum().backward()
    grad = pos.grad.cpu().numpy()
    wn = w.cpu().numpy()
    e = energy.detach().cpu().numpy()
    direct = engine.Batch(mols, accuracy=ACC).run(gradient=True)
    for i, ((z, _), (e_ref, g_ref), r) in enumerate(zip(mols, ref, direct)):
        nat = len(z)
        assert r.status == 0
        assert np.abs(grad[i, :nat] - wn[i] * r.gradient).max() < 1e-12  # the same engine run
        assert abs(e[i] - r.energy) < 1e-12
        assert abs(e[i] - e_ref) < 1e-9, (i, e[i], e_ref)
        assert np.abs(r.gradient - g_ref).max() < 1e-8, (i, np.abs(r.gradient - g_ref).max())
        assert not grad[i, nat:].any()  # padding atoms
    model.close()


def test_backward_matches_central_differences(engine, adjoint):
    import torch

    from axtb_b200.torch_ops import GFN2Energy

    mols, _ = adjoint
    rng = np.random.default_rng(7)
    pick = rng.choice(len(mols), 16, replace=False)
    sub = [mols[i] for i in pick]
    batch = engine.Batch(sub, accuracy=ACC)
    x = torch.tensor(np.concatenate([p for _, p in sub]), dtype=torch.float64, device="cuda", requires_grad=True)
    GFN2Energy.apply(x, batch).sum().backward()
    g = x.grad.cpu().numpy()
    # two random unit directions per molecule, all displaced geometries in one batch
    h = 1e-4
    disp, dirs = [], []
    for z, p in sub:
        for _ in range(2):
            u = rng.normal(size=p.shape)
            u /= np.linalg.norm(u)
            dirs.append(u)
            disp += [(z, p + h * u), (z, p - h * u)]
    e = [r.energy for r in engine.Batch(disp, accuracy=ACC).run(gradient=False)]
    off = np.concatenate([[0], np.cumsum([len(z) for z, _ in sub])])
    for k in range(len(dirs)):
        i = k // 2
        fd = (e[2 * k] - e[2 * k + 1]) / (2 * h)
        an = float((g[off[i] : off[i + 1]] * dirs[k]).sum())
        assert abs(fd - an) < 2e-7, (k, fd, an)
    batch.close()

