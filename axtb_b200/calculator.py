"""Python face of the engine, mirroring axtb's calculator interface.

``Calculator(numbers, positions, charge=0, uhf=None, **options)`` is the counterpart of
``axtb::Calculator::new(Hamiltonian::Gfn2, numbers, positions, charge, uhf, Options)``
(crates/axtb/src/calculator.rs:92-128) and ``Calculator.singlepoint(positions, gradient=True)``
of ``Method::singlepoint`` (crates/base/src/method/mod.rs:62), returning the fields of
``SinglePoint`` (crates/base/src/method/results.rs:39-57). Errors raise ``AxtbError`` with the
kind of crates/base/src/error.rs:8-24. ``Batch`` runs many molecules in one device pass.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib

KINDS = {1: "input", 2: "unsupported_element", 3: "scf_not_converged", 4: "numerical", 5: "device"}
TERM_NAMES = ("repulsion", "dispersion", "electronic", "isotropic_es", "third_order", "anisotropic", "entropy",
              "band")


class AxtbError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{KINDS.get(code, 'error')}: {message}")
        self.code = code
        self.kind = KINDS.get(code, "error")


@dataclass
class SinglePoint:
    energy: float
    gradient: np.ndarray | None
    charges: np.ndarray
    dipole: np.ndarray
    qsh: np.ndarray
    dpat: np.ndarray
    qpat: np.ndarray
    terms: dict = field(default_factory=dict)
    iterations: int = 0
    converged: bool = False
    status: int = 0
    energy_change: float = 0.0
    residual: float = 0.0
    mixer_used: str = "broyden"  # "broyden", "diis" or "diis-fallback" (auto after Broyden failed)
    # the electronic structure (with levels=True): every orbital energy, the occupations of both
    # spins and of the alpha spin, the Fermi levels (NaN: aufbau filling) and the temperature
    emo: np.ndarray | None = None
    focc: np.ndarray | None = None
    focc_alpha: np.ndarray | None = None
    fermi_levels: tuple = (float("nan"), float("nan"))
    electronic_temperature: float = 0.0
    start: str = "guess"        # "previous": started from previous or given moments (ScfReport::start)
    attempts: list = field(default_factory=list)  # [(mixer, iterations, converged)] of the plan
    timings: dict = field(default_factory=dict)   # wall time (s) per phase of the device pass


def _ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class Moments:
    """SCC moments of one molecule (axtb's ScfGuess / ScfData): shell charges, atomic dipoles
    and atomic quadrupoles (xx, xy, yy, xz, yz, zz)."""
    qsh: np.ndarray
    dpat: np.ndarray
    qpat: np.ndarray

    @staticmethod
    def empty(nat: int, nsh: int) -> "Moments":
        return Moments(np.zeros(nsh), np.zeros((nat, 3)), np.zeros((nat, 6)))

    def checked(self, nat: int, nsh: int) -> "Moments":
        w = Moments(np.ascontiguousarray(self.qsh, dtype=np.float64).reshape(-1),
                    np.ascontiguousarray(self.dpat, dtype=np.float64).reshape(-1, 3),
                    np.ascontiguousarray(self.qpat, dtype=np.float64).reshape(-1, 6))
        if w.qsh.size != nsh or w.dpat.shape[0] != nat or w.qpat.shape[0] != nat:
            raise AxtbError(1, f"moments of {w.qsh.size} shells and {w.dpat.shape[0]} atoms for a molecule of "
                               f"{nsh} shells and {nat} atoms")
        return w


def basis_size(numbers):
    z = np.ascontiguousarray(numbers, dtype=np.int32)
    nsh, nao = C.c_int32(), C.c_int32()
    rc = _lib.load().axtb_gpu_basis_size(z.ctypes.data_as(C.POINTER(C.c_int32)), len(z), C.byref(nsh), C.byref(nao))
    if rc != 0:
        raise AxtbError(rc, "unsupported element")
    return nsh.value, nao.value


class _ResultBuffers:
    def __init__(self, nat, nsh, nao=0, views=None):
        """One molecule's output arrays: its own, or `views` (grad, q, dip, qsh, dp, qp, emo, focc,
        focca) into a batch's field-wise arrays."""
        if views is None:
            views = (np.zeros((nat, 3)), np.zeros(nat), np.zeros(3), np.zeros(nsh), np.zeros((nat, 3)),
                     np.zeros((nat, 6)), np.zeros(nao), np.zeros(nao), np.zeros(nao))
        self.grad, self.q, self.dip, self.qsh, self.dp, self.qp, self.emo, self.focc, self.focca = views
        self.nao = nao
        self.res = _lib.AxtbResult()
        self.bind(False)

    def bind(self, levels: bool):
        """Point the result at these buffers (the level arrays only when levels are wanted: they
        cost the engine one more pass and their copy back)."""
        r = self.res
        r.gradient, r.charges, r.dipole = _ptr(self.grad), _ptr(self.q), _ptr(self.dip)
        r.qsh, r.dpat, r.qpat = _ptr(self.qsh), _ptr(self.dp), _ptr(self.qp)
        on = levels and self.nao > 0
        r.emo = _ptr(self.emo) if on else None
        r.focc = _ptr(self.focc) if on else None
        r.focc_alpha = _ptr(self.focca) if on else None
        self.levels = on
        return r

    def result(self, gradient: bool) -> SinglePoint:
        return _single_point(self.res, self.grad.copy() if gradient else None, self.q.copy(), self.dip.copy(),
                             self.qsh.copy(), self.dp.copy(), self.qp.copy(),
                             *((self.emo.copy(), self.focc.copy(), self.focca.copy()) if self.levels else (None,) * 3))


def _single_point(r, grad, q, dip, qsh, dp, qp, emo, focc, focca) -> SinglePoint:
    """A SinglePoint from the ABI result `r` and arrays the caller owns."""
    used = MIXER_USED[r.mixer_used]
    if used == "diis-fallback":
        attempts = [("broyden", r.fallback_iterations, False), ("diis", r.iterations if r.converged else
                                                                r.iterations - r.fallback_iterations,
                                                                bool(r.converged))]
    else:
        attempts = [(used, r.iterations, bool(r.converged))]
    return SinglePoint(energy=r.energy, gradient=grad, charges=q, dipole=dip, qsh=qsh, dpat=dp, qpat=qp,
                       terms=dict(zip(TERM_NAMES, list(r.terms)), solvation=r.solvation),
                       iterations=r.iterations,
                       converged=bool(r.converged), status=r.status, energy_change=r.energy_change,
                       residual=r.residual, mixer_used=used,
                       emo=emo, focc=focc, focc_alpha=focca,
                       fermi_levels=(r.fermi_levels[0], r.fermi_levels[1]),
                       electronic_temperature=r.electronic_temperature,
                       start="previous" if r.warm_start else "guess", attempts=attempts,
                       timings=dict(zip(("setup", "scf", "gradient", "total"), list(r.timings))))


# SCC mixers by name (crates/axtb/src/scf/mixing.rs:202-214: case-insensitive, "pulay" = DIIS;
# None: the conventions' own)
MIXERS = {"auto": 0, "broyden": 1, "diis": 2, "pulay": 2}
# conventions by name (crates/axtb/src/conventions.rs; the xtb 6.7.1 row is not built)
CONVENTIONS = {"axtb": 0, "xtb": 1, "tblite": 2}
MIXER_USED = ("broyden", "diis", "diis-fallback")


def _mixer(name) -> int:
    if name is None:
        return -1
    try:
        return MIXERS[name.lower()]
    except KeyError:
        raise AxtbError(1, f"unknown SCF mixer {name!r} (auto, broyden or diis)") from None


def _conventions(name: str) -> int:
    try:
        return CONVENTIONS[name.lower()]
    except KeyError:
        raise AxtbError(1, f"unknown conventions {name!r} (axtb, xtb or tblite)") from None


# implicit solvation: (model "alpb" | "gbsa", solvent, reference state "gsolv" | "bar1M" | "reference")
SOLVATION_MODELS = {"alpb": 0, "gbsa": 1}
SOLVATION_STATES = {"gsolv": 0, "bar1m": 1, "reference": 2}


def _solvation(spec):
    if spec is None:
        return -1, None, 0
    model, solvent, *state = spec
    try:
        return SOLVATION_MODELS[model.lower()], solvent.encode(), SOLVATION_STATES[(state[0] if state else "gsolv").lower()]
    except KeyError:
        raise AxtbError(1, f"unknown solvation model or state in {spec!r}") from None


def _options(accuracy=1.0, etemp=300.0, max_iter=250, damping=0.4, guess="eeq", precision="fp64", device=0,
             mixer=None, conventions="axtb", solvation=None, dispersion=True, band_max_nao=None,
             grid_min_nao=None):
    model, solvent, state = _solvation(solvation)
    return _lib.default_options(accuracy=float(accuracy), etemp=float(etemp), max_iter=int(max_iter),
                                damping=float(damping), guess=0 if guess == "eeq" else 1,
                                precision={"fp64": 0, "split": 1}[precision], device=int(device),
                                mixer=_mixer(mixer), conventions=_conventions(conventions), solvation=model,
                                solvent=solvent, solvation_state=state, dispersion=1 if dispersion else 0,
                                band_max_nao=-1 if band_max_nao is None else int(band_max_nao),
                                grid_min_nao=-1 if grid_min_nao is None else int(grid_min_nao))


class Calculator:
    """GFN2-xTB calculator of one molecule on the GPU (axtb::Calculator)."""

    def __init__(self, numbers, positions=None, charge=0.0, uhf=None, **options):
        lib = _lib.load()
        self.numbers = np.ascontiguousarray(numbers, dtype=np.int32)
        self.nat = len(self.numbers)
        self.nsh, self.nao = basis_size(self.numbers)
        self._opts = _options(**options)
        h = C.c_void_p()
        rc = lib.axtb_gpu_create(self.numbers.ctypes.data_as(C.POINTER(C.c_int32)), self.nat, float(charge),
                                 -1 if uhf is None else int(uhf), C.byref(self._opts), C.byref(h))
        if rc != 0:
            raise AxtbError(rc, _lib.last_error(None))
        self._h = h
        self._buf = _ResultBuffers(self.nat, self.nsh, self.nao)
        self.positions = None if positions is None else np.asarray(positions, dtype=np.float64).reshape(-1, 3)

    def singlepoint(self, positions=None, gradient=True, levels=True) -> SinglePoint:
        """Energy (+ gradient) at `positions`; `levels`: also every orbital energy and the
        occupations."""
        x = self.positions if positions is None else np.asarray(positions, dtype=np.float64).reshape(-1, 3)
        x = np.ascontiguousarray(x)
        res = self._buf.bind(levels)
        rc = _lib.load().axtb_gpu_singlepoint(self._h, _ptr(x), int(bool(gradient)), C.byref(res))
        if rc != 0:
            raise AxtbError(rc, _lib.last_error(self._h))
        return self._buf.result(gradient)

    def wavefunction(self) -> Moments | None:
        """The moments the next SCF starts from (Method::wavefunction): the last converged
        single point's, or given ones; None when there are none."""
        w = Moments.empty(self.nat, self.nsh)
        rc = _lib.load().axtb_gpu_get_moments(self._h, _ptr(w.qsh), _ptr(w.dpat), _ptr(w.qpat))
        return w if rc == 0 else None

    def set_wavefunction(self, moments: Moments):
        """Start the next SCF from `moments` (Method::set_wavefunction)."""
        self._set(moments, 1)

    def set_history(self, moments: Moments | None):
        """`moments` as this calculator's previous ones, None to forget them
        (Method::set_history)."""
        self._set(moments, 0)

    def _set(self, moments, given):
        lib = _lib.load()
        if moments is None:
            rc = lib.axtb_gpu_set_moments(self._h, None, None, None, given)
        else:
            w = moments.checked(self.nat, self.nsh)
            rc = lib.axtb_gpu_set_moments(self._h, _ptr(w.qsh), _ptr(w.dpat), _ptr(w.qpat), given)
        if rc != 0:
            raise AxtbError(rc, _lib.last_error(self._h))

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().axtb_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many molecules (numbers, positions, charge, uhf) in one device pass."""

    def __init__(self, molecules, **options):
        lib = _lib.load()
        self._keep = []
        self.mols = []
        arr = (_lib.AxtbMol * len(molecules))()
        for i, m in enumerate(molecules):
            z = np.ascontiguousarray(m[0], dtype=np.int32)
            x = np.ascontiguousarray(m[1], dtype=np.float64).reshape(-1, 3)
            q = float(m[2]) if len(m) > 2 else 0.0
            u = m[3] if len(m) > 3 else None
            self._keep += [z, x]
            arr[i].nat = len(z)
            arr[i].numbers = z.ctypes.data_as(C.POINTER(C.c_int32))
            arr[i].positions = _ptr(x)
            arr[i].charge = q
            arr[i].uhf = -1 if u is None else int(u)
            self.mols.append((z, x))
        self._opts = _options(**options)
        b = C.c_void_p()
        rc = lib.axtb_gpu_batch_create(arr, len(molecules), C.byref(self._opts), C.byref(b))
        if rc != 0:
            raise AxtbError(rc, _lib.last_error(None))
        self._b = b
        self.nmol = len(molecules)
        self.natoms = np.array([len(z) for z, _ in self.mols])
        # the outputs field by field over the whole batch (one copy per field after a run), each
        # molecule's ABI result pointing at its rows
        sizes = np.array([basis_size(z) for z, _ in self.mols], dtype=np.int64).reshape(-1, 2)
        self._at = np.concatenate([[0], np.cumsum(self.natoms)])
        self._sh = np.concatenate([[0], np.cumsum(sizes[:, 0])])
        self._ao = np.concatenate([[0], np.cumsum(sizes[:, 1])])
        natT, nshT, naoT = int(self._at[-1]), int(self._sh[-1]), int(self._ao[-1])
        self._all = (np.zeros((natT, 3)), np.zeros(natT), np.zeros((self.nmol, 3)), np.zeros(nshT),
                     np.zeros((natT, 3)), np.zeros((natT, 6)), np.zeros(naoT), np.zeros(naoT), np.zeros(naoT))
        self._bufs = []
        for i in range(self.nmol):
            a, sh, ao = slice(self._at[i], self._at[i + 1]), slice(self._sh[i], self._sh[i + 1]), slice(self._ao[i], self._ao[i + 1])
            g, q, d, qs, dp, qp, emo, focc, focca = self._all
            views = (g[a], q[a], d[i], qs[sh], dp[a], qp[a], emo[ao], focc[ao], focca[ao])
            self._bufs.append(_ResultBuffers(int(self.natoms[i]), int(sizes[i, 0]), int(sizes[i, 1]), views))
        self._res = (_lib.AxtbResult * self.nmol)()
        self._bound = None  # the levels flag the results were last bound with

    def run(self, positions=None, gradient=True, levels=False):
        """Single points of every molecule (positions: list of (nat, 3) arrays or None for the
        set-up geometries); returns a list of SinglePoint (status per molecule). `levels`: also
        every orbital energy and the occupations of each molecule."""
        lib = _lib.load()
        levels = bool(levels)
        if self._bound != levels:  # the pointers stay valid between runs
            for i, bf in enumerate(self._bufs):
                self._res[i] = bf.bind(levels)
            self._bound = levels
        st = np.zeros(self.nmol, dtype=np.int32)
        xp = None
        if positions is not None:
            flat = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.float64).reshape(-1) for p in positions]))
            xp = _ptr(flat)
        rc = lib.axtb_gpu_batch_run(self._b, xp, int(bool(gradient)), self._res, st.ctypes.data_as(C.POINTER(C.c_int32)))
        if rc != 0:
            raise AxtbError(rc, _lib.last_error(None))
        # one copy per field (the gradients and the levels only when asked for), then each
        # molecule's rows as views of the copies
        g, q, d, qs, dp, qp, emo, focc, focca = self._all
        g = g.copy() if gradient else None
        q, d, qs, dp, qp = q.copy(), d.copy(), qs.copy(), dp.copy(), qp.copy()
        if levels:
            emo, focc, focca = emo.copy(), focc.copy(), focca.copy()
        out = []
        at, sh, ao = self._at, self._sh, self._ao
        for i in range(self.nmol):
            a0, a1, s0, s1 = at[i], at[i + 1], sh[i], sh[i + 1]
            lv = (emo[ao[i]:ao[i + 1]], focc[ao[i]:ao[i + 1]], focca[ao[i]:ao[i + 1]]) if levels else (None,) * 3
            out.append(_single_point(self._res[i], g[a0:a1] if gradient else None, q[a0:a1], d[i], qs[s0:s1],
                                     dp[a0:a1], qp[a0:a1], *lv))
        return out

    def run_device(self, d_positions: int, d_energy: int, d_gradient: int, gradient=True):
        """Device-resident run: pointers (ints) to device arrays of positions (natT*3), energies
        (nmol) and gradients (natT*3). Returns the per-molecule status array."""
        st = np.zeros(self.nmol, dtype=np.int32)
        rc = _lib.load().axtb_gpu_batch_run_device(self._b, C.c_void_p(d_positions), int(bool(gradient)),
                                                   C.c_void_p(d_energy), C.c_void_p(d_gradient),
                                                   st.ctypes.data_as(C.POINTER(C.c_int32)))
        if rc != 0:
            raise AxtbError(rc, _lib.last_error(None))
        return st

    def set_restart(self, enable: bool = True, retry_fresh: bool = True):
        """Start later runs from each molecule's converged moments of the previous run (a
        trajectory of geometries); a molecule that then does not converge runs once more from
        the guess (axtb's Calculator under Restart::Previous), unless ``retry_fresh`` is False
        (then it reports the failure, as a displaced point of axtb's numerical Hessian does)."""
        mode = (1 if retry_fresh else 2) if enable else 0
        rc = _lib.load().axtb_gpu_batch_set_restart(self._b, mode)
        if rc != 0:
            raise AxtbError(rc, _lib.last_error(None))

    def get_moments(self, mol: int) -> Moments:
        """Molecule `mol`'s converged output moments of the last run."""
        z, _ = self.mols[mol]
        w = Moments.empty(len(z), basis_size(z)[0])
        rc = _lib.load().axtb_gpu_batch_get_moments(self._b, mol, _ptr(w.qsh), _ptr(w.dpat), _ptr(w.qpat))
        if rc != 0:
            raise AxtbError(rc, _lib.last_error(None))
        return w

    def set_moments(self, mol: int, moments: Moments):
        """Start molecule `mol` of the next run from `moments` (turns restarts on)."""
        z, _ = self.mols[mol]
        w = moments.checked(len(z), basis_size(z)[0])
        rc = _lib.load().axtb_gpu_batch_set_moments(self._b, mol, _ptr(w.qsh), _ptr(w.dpat), _ptr(w.qpat))
        if rc != 0:
            raise AxtbError(rc, _lib.last_error(None))

    def set_profiling(self, enable: bool = True):
        _lib.load().axtb_gpu_batch_set_profiling(self._b, int(bool(enable)))

    def profile(self) -> dict:
        import json

        buf = C.create_string_buffer(1 << 16)
        _lib.load().axtb_gpu_batch_profile(self._b, buf, 1 << 16)
        return json.loads(buf.value.decode())

    @property
    def stream(self) -> int:
        return _lib.load().axtb_gpu_batch_stream(self._b) or 0

    @property
    def launches(self) -> int:
        return int(_lib.load().axtb_gpu_batch_launches(self._b))

    def debug(self, mol: int, what: str) -> np.ndarray:
        z, _ = self.mols[mol]
        nat = len(z)
        nsh, nao = basis_size(z)
        size = {"cn": nat, "eeq": nat, "emo": nao, "focc": nao, "eigen_cycles": 1, "status_bits": 1, "dipole": 3 * nao * nao,
                "quadrupole": 6 * nao * nao}.get(what, nao * nao)
        out = np.zeros(size)
        rc = _lib.load().axtb_gpu_batch_debug(self._b, mol, _lib.DBG[what], _ptr(out))
        if rc != 0:
            raise AxtbError(rc, _lib.last_error(None))
        if what in ("dipole", "quadrupole"):
            k = 3 if what == "dipole" else 6
            return out.reshape(k, nao, nao).transpose(0, 2, 1).copy()
        if size == nao * nao and what not in ("cn", "eeq", "emo", "focc"):
            return out.reshape(nao, nao).T.copy()
        return out

    def close(self):
        if getattr(self, "_b", None):
            _lib.load().axtb_gpu_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
