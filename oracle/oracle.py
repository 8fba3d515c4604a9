"""TEST INFRASTRUCTURE - NOT PART OF THE PRODUCT.

ctypes binding of the C++ oracle (``oracle/gfn2_oracle.cpp``): the CPU FP64 restatement of
axtb's GFN2-xTB energy + gradient (default conventions) that the parity tests, the smoke
check and bench.py's CPU baseline call. Only ``tests/``, ``__graft_entry__.smoke`` and
``bench.py`` (its ``cpu_baseline`` and ``--impl reference`` legs) import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "libgfn2_oracle.so"


class _Run(C.Structure):
    _fields_ = [
        ("nat", C.c_int), ("numbers", C.POINTER(C.c_int)), ("positions", C.POINTER(C.c_double)),
        ("charge", C.c_double), ("uhf", C.c_int), ("accuracy", C.c_double), ("etemp", C.c_double),
        ("max_iter", C.c_int), ("want_gradient", C.c_int), ("eig_backend", C.c_int),
        ("lapack_threads", C.c_int), ("mixer", C.c_int), ("conventions", C.c_int),
        ("solv_model", C.c_int), ("solvent", C.c_char_p), ("solv_state", C.c_int), ("no_dispersion", C.c_int),
        ("energy", C.POINTER(C.c_double)), ("gradient", C.POINTER(C.c_double)),
        ("qat", C.POINTER(C.c_double)), ("qsh", C.POINTER(C.c_double)),
        ("dpat", C.POINTER(C.c_double)), ("qpat", C.POINTER(C.c_double)),
        ("dipole", C.POINTER(C.c_double)), ("terms", C.POINTER(C.c_double)),
        ("emo", C.POINTER(C.c_double)), ("focc", C.POINTER(C.c_double)),
        ("density", C.POINTER(C.c_double)), ("wdensity", C.POINTER(C.c_double)),
        ("e_solvation", C.c_double), ("iterations", C.c_int), ("converged", C.c_int), ("mixer_used", C.c_int), ("nsh", C.c_int),
        ("nao", C.c_int),
        ("error", C.c_char * 256),
    ]


MIXERS = {None: -1, "auto": 0, "broyden": 1, "diis": 2}
CONVENTIONS = {"axtb": 0, "xtb": 1, "tblite": 2}
SOLV_MODELS = {None: -1, "alpb": 0, "gbsa": 1}
SOLV_STATES = {"gsolv": 0, "bar1m": 1, "reference": 2}
MIXER_USED = ("broyden", "diis", "diis-fallback")

TERM_NAMES = ("repulsion", "dispersion", "electronic", "isotropic_es", "third_order", "anisotropic",
              "entropy", "band")


def build() -> Path:
    """Compile the oracle (``make -C oracle``) if its library is missing or stale."""
    src = max((HERE / f).stat().st_mtime for f in ("gfn2_oracle.cpp", "gfn2_oracle.h", "Makefile"))
    if not LIB.exists() or LIB.stat().st_mtime < src:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(str(LIB))
        _lib.oracle_singlepoint.argtypes = [C.POINTER(_Run)]
        _lib.oracle_sizes.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        _lib.oracle_integrals.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_double] + \
            [C.POINTER(C.c_double)] * 5
        _lib.oracle_diis_coefficients.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _lib.oracle_diis_coefficients.restype = None
        _lib.oracle_diis_linear.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                            C.c_double, C.c_int, C.POINTER(C.c_double)]
    return _lib


def diis_coefficients(residuals):
    """Pulay coefficients of the residuals (rows, oldest first) by the oracle's DIIS."""
    r = np.ascontiguousarray(residuals, dtype=np.float64)
    c = np.zeros(r.shape[0])
    lib().oracle_diis_coefficients(r.shape[0], r.shape[1], _p(r), _p(c))
    return c


def diis_linear(eig, b, damp=0.4, tol=1e-12, max_steps=100):
    """DIIS on q = diag(eig) q + b from q = 0: (steps or -1/-2, last input)."""
    e = np.ascontiguousarray(eig, dtype=np.float64)
    bb = np.ascontiguousarray(b, dtype=np.float64)
    q = np.zeros(len(e))
    steps = lib().oracle_diis_linear(len(e), _p(e), _p(bb), float(damp), float(tol), int(max_steps), _p(q))
    return steps, q


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def sizes(numbers):
    z = np.ascontiguousarray(numbers, dtype=np.int32)
    nsh, nao = C.c_int(), C.c_int()
    if lib().oracle_sizes(len(z), z.ctypes.data_as(C.POINTER(C.c_int)), C.byref(nsh), C.byref(nao)) != 0:
        raise ValueError("unsupported element")
    return nsh.value, nao.value


def singlepoint(numbers, positions, charge=0.0, uhf=None, accuracy=1.0, etemp=300.0, max_iter=250,
                gradient=True, matrices=False, lapack=False, lapack_threads=1, mixer=None, failed=False,
                conventions="axtb", solvation=None, dispersion=True):
    """Run the oracle; returns a dict (energy, gradient, qat, qsh, dpat, qpat, dipole, terms, emo,
    focc, iterations, converged, mixer_used[, density, wdensity]). ``mixer``: None (the
    conventions' mixer: auto for axtb, Broyden for xtb and tblite), "auto" (Broyden, then DIIS
    from the start guess), "broyden" or "diis"; ``conventions``: "axtb", "xtb" (6.8.0) or
    "tblite" (0.8.0); ``solvation``: None or (model "alpb" | "gbsa", solvent, state "gsolv" |
    "bar1M" | "reference"); ``dispersion``: False leaves the D4 term out. Raises RuntimeError on a failed SCF
    unless ``failed`` (then the dict of the failed run carries ``status`` and ``error``)."""
    z = np.ascontiguousarray(numbers, dtype=np.int32)
    x = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
    nat = len(z)
    nsh, nao = sizes(z)
    out = {
        "energy": np.zeros(1), "gradient": np.zeros((nat, 3)), "qat": np.zeros(nat), "qsh": np.zeros(nsh),
        "dpat": np.zeros((nat, 3)), "qpat": np.zeros((nat, 6)), "dipole": np.zeros(3), "terms": np.zeros(8),
        "emo": np.zeros(nao), "focc": np.zeros(nao),
    }
    if matrices:
        out["density"] = np.zeros((nao, nao))
        out["wdensity"] = np.zeros((nao, nao))
    r = _Run()
    r.nat = nat
    r.numbers = z.ctypes.data_as(C.POINTER(C.c_int))
    r.positions = _p(x)
    r.charge = float(charge)
    r.uhf = -1 if uhf is None else int(uhf)
    r.accuracy = float(accuracy)
    r.etemp = float(etemp)
    r.max_iter = int(max_iter)
    r.want_gradient = int(bool(gradient))
    r.eig_backend = 1 if lapack else 0
    r.lapack_threads = int(lapack_threads)
    r.mixer = MIXERS[mixer]
    r.conventions = CONVENTIONS[conventions]
    model, solvent, state = solvation if solvation else (None, "", "gsolv")
    r.solv_model = SOLV_MODELS[model]
    r.solvent = solvent.encode()
    r.solv_state = SOLV_STATES[state.lower()]
    r.no_dispersion = 0 if dispersion else 1
    for k in ("energy", "gradient", "qat", "qsh", "dpat", "qpat", "dipole", "terms", "emo", "focc"):
        setattr(r, k, _p(out[k]))
    if matrices:
        r.density = _p(out["density"])
        r.wdensity = _p(out["wdensity"])
    rc = lib().oracle_singlepoint(C.byref(r))
    if rc != 0 and not failed:
        raise RuntimeError(f"oracle status {rc}: {r.error.decode()}")
    out["status"] = rc
    out["error"] = r.error.decode()
    out["mixer_used"] = MIXER_USED[r.mixer_used]
    out["energy"] = float(out["energy"][0])
    out["terms"] = dict(zip(TERM_NAMES, out["terms"].tolist()))
    out["terms"]["solvation"] = r.e_solvation
    out["iterations"] = r.iterations
    out["converged"] = bool(r.converged)
    if matrices:
        # column-major on the C side: transpose the row-major view
        out["density"] = out["density"].T.copy()
        out["wdensity"] = out["wdensity"].T.copy()
    return out


def integrals(numbers, positions, accuracy=1.0):
    """CN, S, H0, D (3), Q (6) of one geometry (matrices as [mu, nu])."""
    z = np.ascontiguousarray(numbers, dtype=np.int32)
    x = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
    nsh, nao = sizes(z)
    cn = np.zeros(len(z))
    S = np.zeros((nao, nao))
    H = np.zeros((nao, nao))
    D = np.zeros((3, nao, nao))
    Q = np.zeros((6, nao, nao))
    rc = lib().oracle_integrals(len(z), z.ctypes.data_as(C.POINTER(C.c_int)), _p(x), float(accuracy),
                                _p(cn), _p(S), _p(H), _p(D), _p(Q))
    if rc != 0:
        raise RuntimeError(f"oracle_integrals status {rc}")
    return cn, S.T.copy(), H.T.copy(), D.transpose(0, 2, 1).copy(), Q.transpose(0, 2, 1).copy()


def lapack_path():
    """The image's OpenBLAS/LAPACK (scipy's bundled build) for the timed baseline, or None."""
    try:
        import scipy
    except ImportError:
        return None
    d = Path(scipy.__file__).resolve().parent.parent / "scipy.libs"
    for f in sorted(d.glob("libscipy_openblas*.so*")):
        return str(f)
    return None


def enable_lapack() -> bool:
    """Point the oracle's optional LAPACK backend at the image's library (before first use)."""
    p = lapack_path()
    if p and "AXTB_ORACLE_LAPACK" not in os.environ:
        os.environ["AXTB_ORACLE_LAPACK"] = p
    return p is not None
