#!/usr/bin/env python3
"""Build the hard-SCF golden fixture from axtb's recorded hard-SCF runs.

axtb's hard-SCF set (``tests/scf_hard_set.py``) holds 84 generated structures where SCFs struggle
(dissociation scans, metal clusters, small-gap and open-shell molecules, ...) as XYZ files in
``tests/scf_hard/`` (Angstrom; charge and unpaired electrons in the comment line), each run at
300 K and a subset also at 0 K, SCF accuracy 1e-4 and at most 250 iterations. Its recorded
results (``bench/results/scf_hard.json``) give, per case and mixer of axtb's default conventions
(``axtb-broyden``, ``axtb-diis`` and ``axtb-auto``: Broyden, then DIIS from the start guess),
whether the SCF converged, the iteration count, the energy and for ``auto`` the mixer that
produced the result. This script converts the structures to bohr the way the hard-set script
does (coordinate x AATOAU of ``tests/reference_matrix/structures.py``) and writes

    tests/golden/scf_hard.json

Run once in a checkout that has the axtb sources::

    python tests/golden/make_scf_hard.py <path-to-axtb-checkout>
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

if len(sys.argv) < 2:
    sys.exit(f"usage: python {Path(__file__).name} <path-to-axtb-checkout>")
REF = Path(sys.argv[1])
OUT = Path(__file__).with_name("scf_hard.json")
METHODS = ("axtb-broyden", "axtb-diis", "axtb-auto")


def read_xyz(path: Path, aatoau: float, z_of) -> dict:
    lines = path.read_text().splitlines()
    nat = int(lines[0].split()[0])
    head = lines[1]
    nums, pos = [], []
    for line in lines[2:2 + nat]:
        f = line.split()
        nums.append(z_of(f[0]))
        pos.append([float(x) * aatoau for x in f[1:4]])
    return {"numbers": nums, "positions": pos, "charge": int(re.search(r"charge=(-?\d+)", head).group(1)),
            "uhf": int(re.search(r"uhf=(\d+)", head).group(1))}


def main() -> None:
    sys.path.insert(0, str(REF / "tests" / "reference_matrix"))
    import structures as S  # noqa: E402  (axtb's numpy structure builders: AATOAU, element symbols)

    rec = json.loads((REF / "bench" / "results" / "scf_hard.json").read_text())
    settings = rec["settings"]
    runs = {}
    for r in rec["runs"]:
        if r["method"] in METHODS:
            keep = {k: r.get(k) for k in ("converged", "iterations", "energy")}
            if r["method"] == "axtb-auto":
                keep["mixer_used"] = r.get("mixer_used")
            runs.setdefault(r["case"], {})[r["method"]] = keep
    out = []
    for c in rec["cases"]:
        mol = read_xyz(REF / "tests" / "scf_hard" / f"{c['structure']}.xyz", S.AATOAU, S.z_of)
        assert mol["charge"] == c["charge"] and mol["uhf"] == c["uhf"]
        out.append(dict(id=c["id"], category=c["category"], etemp=c["etemp"], accuracy=settings["accuracy"],
                        max_iter=settings["max_iter"], **mol, results=runs[c["id"]]))
    OUT.write_text(json.dumps({"source": "axtb bench/results/scf_hard.json (axtb-broyden, axtb-diis, axtb-auto)",
                               "settings": settings, "cases": out}, indent=0))
    print(f"wrote {len(out)} cases to {OUT}")


if __name__ == "__main__":
    main()
