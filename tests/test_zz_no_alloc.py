"""The allocation-free density entry point (axtb_gpu_density_static) against the engine's own
results and an independent generalized eigensolve (GPU).

Some callers cannot allocate device memory: code that runs inside another framework's
stream-ordered memory pool, or under a fixed device-memory budget, where cudaMalloc would
fail or would synchronise the whole device. For them axtb_gpu_density_static computes the
orbital energies, occupations and density of one molecule (up to 256 basis functions) from its
Fock and overlap matrices with all of its scratch in one array inside the library. This test
runs a molecule through the ordinary batch entry points, reads back the last Fock and overlap
matrices with the orbital energies, occupations and density they produced, feeds the two
matrices to the allocation-free entry point through the C ABI and compares its outputs, on
consecutive calls that reuse the shared scratch array (the last one repeating the first
molecule after a different one has left its contents behind); at the documented maximum of 256
basis functions its outputs are also checked against scipy's generalized eigensolver with a
Fermi filling of its own.

This file is named to be collected last, so that a run stopping at its first failure has
already run every other test; it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KB_HARTREE = 3.1668115634564e-6
TOL = 1e-10


def _engine_case(engine, z, x):
    b = engine.Batch([(z, x)], accuracy=1e-6)
    b.run(gradient=False, levels=True)
    case = {k: b.debug(0, k) for k in ("fock", "overlap", "emo", "focc", "density")}
    b.close()
    return case


def _static_call(lib, torch, case):
    nao = len(case["emo"])
    dev = torch.device("cuda:0")
    f = torch.tensor(np.asfortranarray(case["fock"]).ravel(order="F"), dtype=torch.float64, device=dev)
    s = torch.tensor(np.asfortranarray(case["overlap"]).ravel(order="F"), dtype=torch.float64, device=dev)
    emo = torch.full((nao,), np.nan, dtype=torch.float64, device=dev)
    focc = torch.full((nao,), np.nan, dtype=torch.float64, device=dev)
    dens = torch.full((nao * nao,), np.nan, dtype=torch.float64, device=dev)
    st = torch.full((1,), -1, dtype=torch.int32, device=dev)
    nel = float(case["focc"].sum())
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.axtb_gpu_density_static(C.c_void_p(f.data_ptr()), C.c_void_p(s.data_ptr()), nao, nel / 2, nel / 2,
                                     300.0 * KB_HARTREE, C.c_void_p(emo.data_ptr()), C.c_void_p(focc.data_ptr()),
                                     C.c_void_p(dens.data_ptr()), C.c_void_p(st.data_ptr()), C.c_void_p(stream))
    assert rc == 0
    torch.cuda.synchronize(dev)
    return (emo.cpu().numpy(), focc.cpu().numpy(), dens.cpu().numpy().reshape(nao, nao, order="F"),
            int(st.cpu().item()))


def test_density_static_matches_engine(engine):
    import torch

    from axtb_b200 import _lib, structures

    lib = _lib.load()
    a = _engine_case(engine, *structures.water_cluster(8, seed=4))
    b = _engine_case(engine, *structures.alkane(12, seed=2))
    for case in (a, b, a):
        emo, focc, dens, status = _static_call(lib, torch, case)
        assert status == 0
        assert np.abs(emo - case["emo"]).max() < TOL
        assert np.abs(focc - case["focc"]).max() < TOL
        assert np.abs(dens - case["density"]).max() < TOL


def _fermi(eps, nel, kt):
    """Occupations (0..2) of the levels eps holding nel electrons at kT, by bisection on the
    chemical potential (an independent filling, not the engine's Newton iteration)."""
    lo, hi = eps[0] - 10.0, eps[-1] + 10.0
    for _ in range(200):
        mu = 0.5 * (lo + hi)
        f = 2.0 / (1.0 + np.exp(np.clip((eps - mu) / kt, -700, 700)))
        if f.sum() > nel:
            hi = mu
        else:
            lo = mu
    return 2.0 / (1.0 + np.exp(np.clip((eps - 0.5 * (lo + hi)) / kt, -700, 700)))


def test_density_static_at_its_maximum_matches_scipy(engine):
    """C42H86 (254 basis functions, near the 256 limit): orbital energies, occupations and
    density from a plain generalized eigensolve F C = S C e (scipy.linalg.eigh), on two calls."""
    import scipy.linalg
    import torch

    from axtb_b200 import _lib, structures

    lib = _lib.load()
    case = _engine_case(engine, *structures.alkane(42, seed=3))
    nao = len(case["emo"])
    assert 250 <= nao <= 256
    F, S = case["fock"], case["overlap"]
    eps, C = scipy.linalg.eigh(0.5 * (F + F.T), 0.5 * (S + S.T))
    nel = float(case["focc"].sum())
    f = _fermi(eps, nel, 300.0 * KB_HARTREE)
    P = (C * f) @ C.T
    for _ in range(2):
        emo, focc, dens, status = _static_call(lib, torch, case)
        assert status == 0
        assert np.abs(emo - eps).max() < 1e-9
        assert np.abs(focc - f).max() < 1e-8
        assert np.abs(dens - P).max() < 1e-8


def test_density_static_rejects_oversize(engine):
    from axtb_b200 import _lib

    lib = _lib.load()
    rc = lib.axtb_gpu_density_static(C.c_void_p(1), C.c_void_p(1), 257, 1.0, 1.0, 0.0, C.c_void_p(1), C.c_void_p(1),
                                     C.c_void_p(1), None, None)
    assert rc == _lib.AXTB_ERR_INPUT
    assert "256" in _lib.last_error()
