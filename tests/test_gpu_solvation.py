"""Implicit solvation (ALPB, GBSA) on the GPU against axtb's records and the oracle (GPU).

tests/golden/solvation.json: 483 solvated single points of axtb's reference matrix (ALPB and GBSA,
25 solvents and xtb's aliases, gsolv / bar1M / reference states) with axtb's energies; every one
must agree to 1e-9 Eh (one batch per solvent setting), in axtb's own conventions and in its xtb
(483 recorded) and tblite (468) conventions. Gradients against the oracle to
1e-8 Eh/bohr.
"""
import json
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SOLV = json.loads((Path(__file__).parent / "golden" / "solvation.json").read_text())["cases"]


@pytest.mark.parametrize("conv,count", [("axtb", 483), ("xtb", 483), ("tblite", 468)])
def test_solvated_energies_match_axtb_records(engine, conv, count):
    groups = {}
    for c in SOLV:
        if conv == "axtb" or conv in c["conventions"]:
            key = (c["model"], c["solvent"], c["state"], c["accuracy"], c["etemp"], c["max_iter"])
            groups.setdefault(key, []).append(c)
    bad, n = [], 0
    for (model, solvent, state, acc, etemp, max_iter), cases in groups.items():
        mols = [(np.array(c["numbers"]), np.array(c["positions"]), c["charge"], c["uhf"]) for c in cases]
        b = engine.Batch(mols, accuracy=acc, etemp=etemp, max_iter=max_iter, solvation=(model, solvent, state),
                         conventions=conv)
        for c, r in zip(cases, b.run(gradient=False)):
            n += 1
            rec = c if conv == "axtb" else c["conventions"][conv]
            if r.status != 0 or abs(r.energy - rec["energy"]) >= 1e-9:
                bad.append((c["id"], r.status, r.energy - rec["energy"]))
            if conv == "axtb" and abs(r.terms["solvation"] - c["solvation_term"]) >= 1e-9:
                bad.append((c["id"], "solvation term", r.terms["solvation"] - c["solvation_term"]))
        b.close()
    assert n == count and not bad, bad[:10]


@pytest.mark.parametrize("solvation", [("alpb", "water", "gsolv"), ("gbsa", "ch2cl2", "reference"),
                                       ("alpb", "dmso", "bar1M")])
@pytest.mark.parametrize("cid", ["struct-caffeine", "struct-ferrocene", "struct-taxol"])
def test_solvated_singlepoint_matches_oracle(engine, golden, solvation, cid):
    from oracle import oracle as O

    c = golden[cid]
    z, x = np.array(c["numbers"]), np.array(c["positions"])
    r = engine.Calculator(z, x, charge=c["charge"], uhf=c["uhf"], accuracy=1e-6, solvation=solvation).singlepoint(x)
    ref = O.singlepoint(z, x, c["charge"], c["uhf"], accuracy=1e-6, solvation=solvation)
    assert r.converged
    assert abs(r.energy - ref["energy"]) < 1e-9, (r.energy, ref["energy"])
    assert np.abs(r.gradient - ref["gradient"]).max() < 1e-8
    assert np.abs(r.charges - ref["qat"]).max() < 1e-7
    assert abs(r.terms["solvation"] - ref["terms"]["solvation"]) < 1e-9


def test_unknown_solvent_is_an_input_error(engine):
    with pytest.raises(engine.AxtbError) as e:
        engine.Calculator([8, 1, 1], solvation=("alpb", "vacuum"))
    assert e.value.kind == "input"
    with pytest.raises(engine.AxtbError):
        engine.Calculator([8, 1, 1], solvation=("cosmo", "water"))
