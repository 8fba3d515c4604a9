"""Autotuner of the dense-algebra schedule: which molecules use which reduction, and which run
on the whole GPU.

The engine's eigen phase has two schedule choices, both exact (the results agree to
round-off): the tridiagonal reduction of a one-CTA molecule (two-stage: band reduction on
GEMMs, then bulge chasing; or one-stage Householder with the trailing matrix streamed per
column), chosen by the size ``band_max_nao`` below which the two-stage one is used (from 34 AOs:
a smaller matrix already is a band, and keeps the one-stage reduction; measured on
B200: it wins only for small molecules, where the one-stage reduction's per-column chain is
short of work, not for large ones, where its bulge chasing waits on one global-memory round per
block); and the size
``grid_min_nao`` from which a molecule's dense algebra runs on the whole cooperative grid
instead of one CTA. The best crossovers depend on the GPU and the batch, so they are measured:

* ``band_max_nao``: one profiled run of a sample batch with each reduction; the engine's
  per-molecule cycle counters of the eigen phase (the on-chip bulge chasing counted in units of
  the team kernel's half-SM CTAs) are binned by AO count, and the bin edge that minimises the
  sample's total with the two-stage reduction below it is the candidate; it, the default and 0
  (one-stage only) are then timed as whole runs of the sample, and the fastest is kept;
* ``grid_min_nao``: whole runs of the sample with each candidate threshold below its largest
  molecule, timed with CUDA events; the fastest wins (no candidate applies to a sample without
  molecules that large, and the default stays).

``schedule()`` returns the options to pass to ``Batch`` / ``Calculator`` (the cached result for
this GPU, or the defaults), ``tune()`` measures and caches.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np

DEFAULT = {"band_max_nao": 64, "grid_min_nao": 1024}
GRID_CANDIDATES = (512, 768, 1024, 1536, 2048)


def _cache_path() -> Path:
    base = os.environ.get("AXTB_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "axtb_b200")
    return Path(base) / "schedule.json"


def _device_key(device: int) -> str:
    import torch

    p = torch.cuda.get_device_properties(device)
    return f"{p.name}/{p.multi_processor_count}SM"


def schedule(device: int = 0) -> dict:
    """The tuned options of this GPU (band_max_nao, grid_min_nao), or the defaults."""
    try:
        data = json.loads(_cache_path().read_text())
        return dict(data[_device_key(device)]["options"])
    except Exception:
        return dict(DEFAULT)


def crossover(nao: np.ndarray, cyc_two: np.ndarray, cyc_one: np.ndarray, width: int = 32) -> tuple[int, list]:
    """The AO count below which the two-stage reduction is used: of the bin edges (bins of `width`
    AOs), the one that minimises the sample's total eigen cycles with the two-stage reduction below
    it and the one-stage reduction from it on (0 when no edge beats the one-stage reduction
    everywhere); and the bins (lo, hi, n, mean two-stage cycles, mean one-stage cycles)."""
    nao = np.asarray(nao)
    cyc_two, cyc_one = np.asarray(cyc_two, dtype=float), np.asarray(cyc_one, dtype=float)
    lo = (nao // width) * width
    bins = []
    for b in sorted(set(lo.tolist())):
        sel = lo == b
        bins.append((int(b), int(b + width), int(sel.sum()), float(np.mean(cyc_two[sel])), float(np.mean(cyc_one[sel]))))
    best, cut, run = 0.0, 0, 0.0
    for b in bins:  # running sum of the saving (two - one) over the bins below each upper edge
        run += b[2] * (b[3] - b[4])
        if run < best:
            best, cut = run, b[1]
    return int(cut), bins


def _eigen_cycles(mols, options, device):
    from .calculator import Batch

    b = Batch(mols, device=device, **options)
    try:
        b.run(gradient=False)  # warm-up
        b.set_profiling(True)
        b.run(gradient=False)
        cyc = np.array([float(b.debug(i, "eigen_cycles")[0]) for i in range(len(mols))])
        b.set_profiling(False)
    finally:
        b.close()
    return cyc


def _timed_run(mols, options, device, reps=2):
    import torch

    from .calculator import Batch

    b = Batch(mols, device=device, **options)
    try:
        b.run(gradient=True)
        torch.cuda.synchronize(device)
        best = float("inf")
        stream = torch.cuda.ExternalStream(b.stream, device=torch.device("cuda", device))
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.run(gradient=True)
            e1.record(stream)
            torch.cuda.synchronize(device)
            best = min(best, e0.elapsed_time(e1) / 1e3)
    finally:
        b.close()
    return best


def tune(molecules=None, device: int = 0, accuracy: float = 0.1, save: bool = True) -> dict:
    """Measure the schedule on a sample (default: 256 molecules of the mixed benchmark batch) and
    cache it for this GPU; returns {"options": {...}, "bins": [...], "grid_times": {...}}."""
    from . import structures
    from .calculator import basis_size

    mols = molecules if molecules is not None else structures.mixed_batch(256, seed=12345)
    nao = np.array([basis_size(m[0])[1] for m in mols])
    grid = DEFAULT["grid_min_nao"]
    small = [m for m, n in zip(mols, nao) if n < grid]
    nsmall = np.array([n for n in nao if n < grid])
    opts = {"accuracy": accuracy, "grid_min_nao": grid}
    band = DEFAULT["band_max_nao"]
    bins = []
    band_times = {}
    if small:
        two = _eigen_cycles(small, dict(opts, band_max_nao=1 << 30), device)
        one = _eigen_cycles(small, dict(opts, band_max_nao=0), device)
        cut, bins = crossover(nsmall, two, one)
        # the per-molecule cycles do not see the launches' tails (the two-stage eigen phase is
        # three launches, each balanced on its own): the cut, the default and none are timed as
        # whole runs of the sample, and the fastest wins
        for bm in sorted({0, DEFAULT["band_max_nao"], cut}):
            band_times[bm] = _timed_run(mols, {"accuracy": accuracy, "band_max_nao": bm, "grid_min_nao": grid}, device)
        band = min(band_times, key=band_times.get)
    grid_times = {}
    cands = [g for g in GRID_CANDIDATES if g <= int(nao.max())]
    if cands:
        for g in cands + [1 << 30]:
            grid_times[g] = _timed_run(mols, {"accuracy": accuracy, "band_max_nao": band, "grid_min_nao": g}, device)
        grid = min(grid_times, key=grid_times.get)
        if grid == 1 << 30:
            grid = max(int(nao.max()) + 1, DEFAULT["grid_min_nao"])
    result = {"options": {"band_max_nao": int(band), "grid_min_nao": int(grid)}, "bins": bins,
              "band_times": {str(k): v for k, v in band_times.items()},
              "grid_times": {str(k): v for k, v in grid_times.items()}, "sample": len(mols)}
    if save:
        path = _cache_path()
        path.parent.mkdir(parents=True, exist_ok=True)
        try:
            data = json.loads(path.read_text())
        except Exception:
            data = {}
        data[_device_key(device)] = result
        path.write_text(json.dumps(data, indent=1))
    return result
