"""The oracle's implicit solvation (ALPB, GBSA) against axtb's recorded results (CPU).

tests/golden/solvation.json (from axtb's reference matrix, category solvation) holds 483 solvated
single points (ALPB and GBSA, 25 solvents and xtb's aliases, the gsolv, bar1M and reference states)
with axtb's energies in its default conventions at SCF accuracy 1e-6. The oracle must reproduce
every energy to 1e-9 Eh, and its gradient must match central finite differences (h = 1e-4 bohr)
within axtb's consistency bound (2e-7 Eh/bohr; the surface integral drops grid points below a
1e-6 weight, so the energy is smooth only to ~1e-11 Eh).
"""
import json
import multiprocessing as mp
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

SOLV = json.loads((Path(__file__).parent / "golden" / "solvation.json").read_text())["cases"]


def _run(job):
    c, conv = job
    r = O.singlepoint(c["numbers"], c["positions"], c["charge"], c["uhf"], c["accuracy"], c["etemp"], c["max_iter"],
                      gradient=False, failed=True, solvation=(c["model"], c["solvent"], c["state"]), conventions=conv)
    rec = c if conv == "axtb" else c["conventions"][conv]
    return c["id"], r["status"], r["energy"] - rec["energy"], r["iterations"] == rec["iterations"]


@pytest.mark.parametrize("conv,count", [("axtb", 483), ("xtb", 483), ("tblite", 468)])
def test_solvated_energies_match_axtb_records(conv, count):
    """axtb's own runs in each of its conventions (the xtb conventions take xtb 6.8.0's solvation
    variant, the others the corrected one)."""
    jobs = [(c, conv) for c in SOLV if conv == "axtb" or conv in c["conventions"]]
    with mp.get_context("spawn").Pool(min(16, mp.cpu_count())) as pool:
        res = pool.map(_run, jobs, chunksize=4)
    assert len(res) == count
    bad = [r for r in res if r[1] != 0 or abs(r[2]) >= 1e-9]
    assert not bad, bad[:10]
    assert sum(r[3] for r in res) >= 0.98 * len(res)
    # both models and all reference states are covered
    assert {(c["model"], c["state"]) for c in SOLV} == {(m, s) for m in ("alpb", "gbsa")
                                                         for s in ("gsolv", "bar1M", "reference")}


def test_solvation_term_matches_axtb_records():
    """The reported solvation term (surface, shift and polar parts; crates/axtb/src/calculator.rs:314)."""
    worst = 0.0
    for c in SOLV:
        r = O.singlepoint(c["numbers"], c["positions"], c["charge"], c["uhf"], c["accuracy"], c["etemp"],
                          c["max_iter"], gradient=False, solvation=(c["model"], c["solvent"], c["state"]))
        worst = max(worst, abs(r["terms"]["solvation"] - c["solvation_term"]))
    assert worst < 1e-9, worst
    r = O.singlepoint([8, 1, 1], [[0, 0, 0], [0, 1.4, 1.1], [0, -1.4, 1.1]], gradient=False)
    assert r["terms"]["solvation"] == 0.0


@pytest.mark.parametrize("solvation", [("alpb", "water", "gsolv"), ("gbsa", "water", "bar1M"),
                                       ("alpb", "ch2cl2", "reference")])
def test_solvated_gradient_finite_differences(golden, solvation):
    c = golden["struct-caffeine"]
    z, x = c["numbers"], np.array(c["positions"])
    kw = dict(charge=c["charge"], uhf=c["uhf"], accuracy=1e-8, etemp=c["etemp"], solvation=solvation)
    g = O.singlepoint(z, x, **kw)["gradient"]
    h = 1e-4
    for i, k in [(0, 0), (3, 1), (7, 2), (11, 0), (13, 1)]:
        xp, xm = x.copy(), x.copy()
        xp[i, k] += h
        xm[i, k] -= h
        fd = (O.singlepoint(z, xp, gradient=False, **kw)["energy"] - O.singlepoint(z, xm, gradient=False, **kw)["energy"]) / (2 * h)
        assert abs(fd - g[i, k]) < 2e-7, (solvation, i, k, fd, g[i, k])


def test_unknown_solvent_is_an_input_error(golden):
    c = golden["struct-water"]
    r = O.singlepoint(c["numbers"], c["positions"], gradient=False, failed=True, solvation=("alpb", "vacuum", "gsolv"))
    assert r["status"] == 1 and "solvent" in r["error"]
    # xtb's aliases, any case
    e1 = O.singlepoint(c["numbers"], c["positions"], gradient=False, solvation=("gbsa", "CHCl3", "gsolv"))["energy"]
    e2 = O.singlepoint(c["numbers"], c["positions"], gradient=False, solvation=("gbsa", "chloroform", "gsolv"))["energy"]
    assert e1 == e2
