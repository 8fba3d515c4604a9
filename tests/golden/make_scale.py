#!/usr/bin/env python3
"""Oracle results for the at-scale parity tests: the benchmark's large single points.

The molecules are the seeded workload builders of ``axtb_b200/structures.py``:

* (H2O)500: 1500 atoms, 3000 AOs, the 10x10x5 lattice rule, seed 0;
* C200H402: 602 atoms, 1202 AOs, seed 0, 10 % of the dihedrals gauche;
* (H2O)1000: 3000 atoms, 6000 AOs, the 10x10x10 lattice rule, seed 0.

Each is run through the CPU oracle (FP64, axtb's default conventions, LAPACK eigensolver on
all host threads) at SCF accuracy ``ACC``; the file keeps the energy, the energy terms, the
gradient, the Mulliken charges, the iteration count and a checksum of the positions (so a
test notices when the builder no longer makes the same molecule). Run on a CPU box::

    python tests/golden/make_scale.py            # writes tests/golden/scale.npz

It takes about ten minutes on 8 cores, nearly all of it in (H2O)1000.
"""
from __future__ import annotations

import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from axtb_b200 import structures  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).with_name("scale.npz")
ACC = 1e-3  # SCF thresholds 1e-9 Eh and 2e-8 e: the converged energies are stable far below 1e-9 Eh


def cases():
    return {
        "w500": structures.water_cluster(500, seed=0, dims=(10, 10, 5)),
        "c200": structures.alkane(200, seed=0, gauche=0.1),
        "w1000": structures.water_cluster(1000, seed=0, dims=(10, 10, 10)),
    }


def checksum(x: np.ndarray) -> float:
    w = np.arange(1, x.size + 1, dtype=np.float64)
    return float(np.dot(w, x.reshape(-1)))


def main() -> None:
    O.enable_lapack()
    threads = os.cpu_count() or 1
    out = {"accuracy": np.float64(ACC)}
    for name, (z, x) in cases().items():
        t0 = time.time()
        r = O.singlepoint(z, x, accuracy=ACC, lapack=True, lapack_threads=threads)
        print(f"{name}: {len(z)} atoms, E = {r['energy']:.12f}, {r['iterations']} iterations, "
              f"{time.time() - t0:.0f} s", flush=True)
        out[f"{name}_natoms"] = np.int64(len(z))
        out[f"{name}_xsum"] = np.float64(checksum(x))
        out[f"{name}_energy"] = np.float64(r["energy"])
        out[f"{name}_gradient"] = r["gradient"]
        out[f"{name}_qat"] = r["qat"]
        out[f"{name}_iterations"] = np.int64(r["iterations"])
        out[f"{name}_terms"] = np.array([r["terms"][k] for k in O.TERM_NAMES])
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
