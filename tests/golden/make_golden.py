#!/usr/bin/env python3
"""Build the golden fixtures of the parity tests from axtb's reference matrix.

axtb records, for every case of its reference matrix, the inputs (generated by the numpy
builders in ``tests/reference_matrix/{cases,structures}.py``) and the results of axtb 0.1.0
in its default conventions (``tests/reference_matrix/results.json``: ``programs.axtb`` with the
energy, the energy terms, Mulliken charges, dipole and SCF iterations, at SCF accuracy 1e-6).
This script re-runs the builders (plain numpy, importable without axtb itself), keeps the
gas-phase cases with dispersion that the GFN2 E+grad path covers (categories elements,
structures, multielement, charges, spin, etemp_acc, open_shell_metals, threads) and writes

    tests/golden/reference_matrix.json

with numbers, positions (bohr), charge, uhf, accuracy, etemp, max_iter and the recorded axtb
results, plus axtb's energies and iterations in its xtb (6.8.0) and tblite (0.8.0) conventions
(``programs["axtb[xtb]"]``, ``programs["axtb[tblite]"]``); and, in

    tests/golden/solvation.json

the cases of the solvation category (ALPB or GBSA, solvent, reference state) with axtb's recorded
energies. Run once in a checkout that has the axtb sources::

    python tests/golden/make_golden.py <path-to-axtb-checkout>
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

if len(sys.argv) < 2:
    sys.exit(f"usage: python {Path(__file__).name} <path-to-axtb-checkout>")
REF = Path(sys.argv[1])
OUT = Path(__file__).with_name("reference_matrix.json")
SOLV = Path(__file__).with_name("solvation.json")
KEEP = {"elements", "structures", "multielement", "charges", "spin", "etemp_acc", "open_shell_metals", "threads"}


def main() -> None:
    sys.path.insert(0, str(REF / "tests" / "reference_matrix"))
    import cases as C  # noqa: E402  (axtb's numpy case builders)

    results = json.loads((REF / "tests" / "reference_matrix" / "results.json").read_text())["cases"]
    out = []
    for name in sorted(KEEP):
        for c in C.CATEGORIES[name]():
            r = results.get(c["id"])
            if r is None:
                continue
            ax = r.get("programs", {}).get("axtb")
            if not ax or not ax.get("ok") or "energy" not in ax:
                continue
            if any(k in c for k in ("alpb", "gbsa", "solvation_state")) or c.get("dispersion") is False:
                continue
            out.append({
                "id": c["id"],
                "category": name,
                "numbers": c["numbers"],
                "positions": c["positions"],
                "charge": c["charge"],
                "uhf": c["uhf"],
                "accuracy": c.get("accuracy", 1.0),
                "etemp": c.get("etemp", 300.0),
                "max_iter": c.get("max_iter", 250),
                "energy": ax["energy"],
                "terms": ax.get("terms"),
                "charges": ax.get("charges"),
                "dipole": ax.get("dipole"),
                "iterations": ax.get("iterations"),
                # axtb 0.1.0 in its xtb (6.8.0) and tblite (0.8.0) conventions, where it ran
                "conventions": {k: {"energy": r["programs"][p]["energy"],
                                    "iterations": r["programs"][p].get("iterations")}
                                for k, p in (("xtb", "axtb[xtb]"), ("tblite", "axtb[tblite]"))
                                if r["programs"].get(p, {}).get("ok") and "energy" in r["programs"][p]},
            })
    OUT.write_text(json.dumps({"source": "axtb tests/reference_matrix/results.json (programs.axtb)",
                               "cases": out}, indent=0))
    print(f"wrote {len(out)} cases to {OUT}")
    # implicit solvation (category solvation): ALPB or GBSA, solvent, reference state (gsolv when
    # the case names none), axtb's recorded energy in its default conventions
    solv = []
    for c in C.CATEGORIES["solvation"]():
        r = results.get(c["id"])
        ax = (r or {}).get("programs", {}).get("axtb")
        if not ax or not ax.get("ok") or "energy" not in ax:
            continue
        model = "alpb" if "alpb" in c else "gbsa"
        solv.append({
            "id": c["id"], "numbers": c["numbers"], "positions": c["positions"], "charge": c["charge"],
            "uhf": c["uhf"], "accuracy": c.get("accuracy", 1.0), "etemp": c.get("etemp", 300.0),
            "max_iter": c.get("max_iter", 250), "model": model, "solvent": c[model],
            "state": c.get("solvation_state") or "gsolv", "energy": ax["energy"],
            "iterations": ax.get("iterations"), "solvation_term": (ax.get("terms") or {}).get("solvation"),
            "conventions": {k: {"energy": r["programs"][p]["energy"], "iterations": r["programs"][p].get("iterations")}
                            for k, p in (("xtb", "axtb[xtb]"), ("tblite", "axtb[tblite]"))
                            if r["programs"].get(p, {}).get("ok") and "energy" in r["programs"][p]},
        })
    SOLV.write_text(json.dumps({"source": "axtb tests/reference_matrix/results.json (programs.axtb, "
                                          "category solvation)", "cases": solv}, indent=0))
    print(f"wrote {len(solv)} cases to {SOLV}")


if __name__ == "__main__":
    main()
