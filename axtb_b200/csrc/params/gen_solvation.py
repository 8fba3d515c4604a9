#!/usr/bin/env python3
"""Generate solvation_tables.h (ALPB/GBSA parameters of GFN2-xTB) from axtb's solvation crate.

Reads ``crates/solvation/src/params.rs`` (the GFN2 ALPB and GBSA parameter sets of xtb's
``param_{alpb,gbsa}_*.fh``, the solvent-name aliases, the D3 van der Waals radii and the model
constants) and ``crates/solvation/src/lebedev_data.rs`` (the Lebedev-Laikov generators), and
writes the parameter sets, the name tables and the default 230-point angular grid. The grid is
expanded from its Oh generators in xtb's point order (``lebedev.f90`` genOh1..genOh6), so that
surface sums run in the reference's order. Run once in a checkout that has the axtb sources::

    python axtb_b200/csrc/params/gen_solvation.py <path-to-axtb-checkout>
"""
from __future__ import annotations

import math
import re
import sys
from pathlib import Path

if len(sys.argv) < 2:
    sys.exit(f"usage: python {Path(__file__).name} <path-to-axtb-checkout>")
REF = Path(sys.argv[1])
OUT = Path(__file__).with_name("solvation_tables.h")
SRC = REF / "crates" / "solvation" / "src"
DEFAULT_GRID = 230

CONSTANTS = ["NELEM", "AUTOAA", "AUTOKCAL", "KB", "MOLCM3TOAU", "SURFACE_TENSION", "LRCUT_AA", "SRCUT_AA",
             "REF_DENSITY", "REF_MOLECULAR_MASS", "IDEAL_GAS_MOL_VOLUME", "AMBIENT_TEMPERATURE",
             "DEFAULT_TEMPERATURE", "ALPB_ALPHA", "SMOOTH_W_AA", "TOLSESP", "ZETA_P16", "OBC_ALPHA", "OBC_BETA",
             "OBC_GAMMA"]


def strip_comments(text: str) -> str:
    return re.sub(r"//[^\n]*", "", text)


def number_list(body: str) -> list[float]:
    return [float(x) for x in re.findall(r"[-+]?\d+\.?\d*(?:[eE][-+]?\d+)?", body)]


def parse_params(text: str):
    consts = {}
    for name in CONSTANTS:
        m = re.search(rf"pub const {name}: \w+ = ([^;]+);", text)
        consts[name] = m.group(1).strip()
    sets = {}
    for m in re.finditer(r"pub static (GFN2_\w+): RawParam = RawParam \{(.*?)\n\};", text, re.S):
        body = m.group(2)
        p = {"name": re.search(r'name: "([^"]+)"', body).group(1)}
        for key in ("epsv", "smass", "rhos", "c1", "rprobe", "gshift", "soset"):
            p[key] = float(re.search(rf"\b{key}: ([-+0-9.eE]+),", body).group(1))
        for key in ("gamscale", "sx", "tmp"):
            arr = re.search(rf"\b{key}: \[(.*?)\]", body, re.S).group(1)
            p[key] = number_list(arr)
            assert len(p[key]) == 94, (m.group(1), key, len(p[key]))
        sets[m.group(1)] = p

    def table(name):
        body = re.search(rf"pub static {name}: &\[\(&str, &RawParam\)\] = &\[(.*?)\n\];", text, re.S).group(1)
        return re.findall(r'\("([^"]+)", &(\w+)\)', body)

    alias_body = re.search(r"pub static NORMALIZE: &\[\(&str, &str\)\] = &\[(.*?)\n\];", text, re.S).group(1)
    aliases = re.findall(r'\("([^"]+)", "([^"]+)"\)', alias_body)
    vdw = number_list(re.search(r"pub static VDW_RAD_D3_AA: \[f64; NELEM\] = \[(.*?)\];", text, re.S).group(1))
    assert len(vdw) == 94
    return consts, sets, table("GFN2_ALPB"), table("GFN2_GBSA"), aliases, vdw


def lebedev(text: str, npoints: int):
    sizes = [int(x) for x in re.search(r"GRID_SIZE: \[usize; \d+\] = \[([^\]]*)\]", text).group(1).split(",")]
    body = text[text.index("pub static GRIDS"):]
    grids = re.findall(r"&\[(.*?)\]", body[body.index("= [") + 3:], re.S)
    gens = re.findall(r"(Oh\d)\(([^)]*)\)", grids[sizes.index(npoints)])
    pts = []
    for kind, args in gens:
        a = [float(x) for x in args.split(",")]
        if kind == "Oh1":
            v, s = a[0], 1.0
            block = [(s, 0, 0), (-s, 0, 0), (0, s, 0), (0, -s, 0), (0, 0, s), (0, 0, -s)]
        elif kind == "Oh2":
            v, s = a[0], math.sqrt(0.5)
            block = [(0, s, s), (0, -s, s), (0, s, -s), (0, -s, -s), (s, 0, s), (-s, 0, s), (s, 0, -s),
                     (-s, 0, -s), (s, s, 0), (-s, s, 0), (s, -s, 0), (-s, -s, 0)]
        elif kind == "Oh3":
            v, s = a[0], math.sqrt(1.0 / 3.0)
            block = [(x, y, z) for z in (s, -s) for y in (s, -s) for x in (s, -s)]
        elif kind == "Oh4":
            s, v = a
            b = math.sqrt(1.0 - 2.0 * s * s)
            block = ([(x, y, zb) for zb in (b, -b) for y in (s, -s) for x in (s, -s)] +
                     [(x, yb, z) for z in (s, -s) for yb in (b, -b) for x in (s, -s)] +
                     [(xb, y, z) for z in (s, -s) for y in (s, -s) for xb in (b, -b)])
        elif kind == "Oh5":
            s, v = a
            b = math.sqrt(1.0 - s * s)
            block = ([(x, y, 0) for y in (b, -b) for x in (s, -s)] + [(x, y, 0) for y in (s, -s) for x in (b, -b)] +
                     [(x, 0, z) for z in (b, -b) for x in (s, -s)] + [(x, 0, z) for z in (s, -s) for x in (b, -b)] +
                     [(0, y, z) for z in (b, -b) for y in (s, -s)] + [(0, y, z) for z in (s, -s) for y in (b, -b)])
        else:
            s, t, v = a
            c = math.sqrt(1.0 - s * s - t * t)
            block = []
            for (p, q, r) in ((s, t, c), (s, c, t), (t, s, c), (t, c, s), (c, s, t), (c, t, s)):
                block += [(x, y, z) for z in (r, -r) for y in (q, -q) for x in (p, -p)]
        pts += [(x, y, z, v) for x, y, z in block]
    assert len(pts) == npoints, len(pts)
    return pts


def main() -> None:
    consts, sets, alpb, gbsa, aliases, vdw = parse_params(strip_comments((SRC / "params.rs").read_text()))
    grid = lebedev(strip_comments((SRC / "lebedev_data.rs").read_text()), DEFAULT_GRID)
    names = sorted(sets)
    idx = {n: i for i, n in enumerate(names)}
    f = lambda x: repr(float(x))
    out = ["// Generated by gen_solvation.py from axtb's solvation crate (LGPL-3.0-or-later); do not edit.",
           "// GFN2-xTB ALPB and GBSA parameters of xtb, D3 van der Waals radii, model constants and the",
           "// 230-point Lebedev-Laikov grid in xtb's point order.", "#pragma once", "", "namespace solvtab {", ""]
    for k in CONSTANTS:
        ctype = "int" if k == "NELEM" else "double"
        out.append(f"constexpr {ctype} {k} = {consts[k]};")
    out += ["", "struct SolventParam {", "    const char* name;",
            "    double epsv, smass, rhos, c1, rprobe, gshift, soset;",
            "    double gamscale[94], sx[94], tmp[94];", "};", "",
            f"static const SolventParam PARAMS[{len(names)}] = {{"]
    for n in names:
        p = sets[n]
        out.append(f'    {{"{p["name"]}", {", ".join(f(p[k]) for k in ("epsv", "smass", "rhos", "c1", "rprobe", "gshift", "soset"))},')
        for key in ("gamscale", "sx", "tmp"):
            out.append("     {" + ", ".join(f(x) for x in p[key]) + "},")
        out.append("    },")
    out.append("};")
    for tname, tab in (("ALPB_SOLVENTS", alpb), ("GBSA_SOLVENTS", gbsa)):
        out.append(f"static const struct {{ const char* name; int param; }} {tname}[{len(tab)}] = {{")
        out += [f'    {{"{s}", {idx[p]}}},' for s, p in tab]
        out.append("};")
    out.append(f"static const struct {{ const char* alias; const char* name; }} ALIASES[{len(aliases)}] = {{")
    out += [f'    {{"{a}", "{b}"}},' for a, b in aliases]
    out.append("};")
    out.append("static const double VDW_RAD_D3_AA[94] = {" + ", ".join(f(x) for x in vdw) + "};")
    out.append(f"static const double LEBEDEV_{DEFAULT_GRID}[{DEFAULT_GRID}][4] = {{")
    out += ["    {" + ", ".join(f(x) for x in p) + "}," for p in grid]
    out += ["};", "", "}  // namespace solvtab", ""]
    OUT.write_text("\n".join(out))
    print(f"wrote {OUT}: {len(names)} parameter sets, {len(alpb)} ALPB and {len(gbsa)} GBSA names, "
          f"{len(aliases)} aliases")


if __name__ == "__main__":
    main()
