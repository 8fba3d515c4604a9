#!/usr/bin/env python3
"""Generate ``gfn2_tables.h``: the GFN2-xTB, STO-nG, EEQ-2019, element and D4 parameter
tables as C arrays.

The tables are the published parametrisations (GFN2-xTB: Bannwarth, Ehlert, Grimme, JCTC 15,
1652 (2019); DFT-D4: Caldeweyher et al., JCP 150, 154122 (2019); EEQ-2019 and STO-nG
expansions), read from the Rust sources of axtb where they are stored as literal arrays:

* ``crates/axtb/src/param/gfn2_data.rs``  (GFN2-xTB element and shell parameters)
* ``crates/axtb/src/param/sto_data.rs``   (STO-nG exponents and coefficients)
* ``crates/axtb/src/param/eeq_data.rs``   (EEQ-2019 parameters of the start guess)
* ``crates/base/src/elements.rs``         (Pauling EN, Pyykko-Atsumi covalent radii)
* ``crates/d4/src/data.rs``               (D4 reference systems and polarisabilities)

Every element expression (``-0.05 * EVTOAU``, ``1.0 + 0.1972612``) is evaluated here in IEEE
double arithmetic, which rounds exactly as the Rust constant evaluation does, and written with
``repr`` (shortest round-trip), so each C value carries the same bits as the reference's.

Run from the repository root::

    python axtb_b200/csrc/params/gen_params.py <path-to-axtb-checkout>

The output header is committed; the script only needs the axtb sources to regenerate it.
"""
from __future__ import annotations

import math
import re
import sys
from pathlib import Path

if len(sys.argv) < 2:
    sys.exit(f"usage: python {Path(__file__).name} <path-to-axtb-checkout>")
REF = Path(sys.argv[1])
OUT = Path(__file__).with_name("gfn2_tables.h")

EVTOAU = 1.0 / 27.21138505
# mctc-lib's Angstrom-to-bohr factor from CODATA 2018 (crates/base/src/units.rs:66-77), evaluated in
# the same double-precision operations; xtb 6.8.0's tables are converted with it
_HBAR_2018 = 6.62607015e-34 / (2.0 * math.pi)
MCTC_AATOAU = 1.0 / (_HBAR_2018 / (9.1093837015e-31 * 299792458.0 * 7.2973525693e-3) * 1e10)
NAMES = {"EVTOAU": EVTOAU, "XTB_AATOAU": MCTC_AATOAU}

SOURCES = {
    "crates/axtb/src/param/gfn2_data.rs": [
        "REP_ALPHA", "REP_ZEFF", "HUBBARD_PARAMETER", "SHELL_HUBBARD", "P_HUBBARD_DERIVS",
        "P_SHPOLY", "P_KCN", "REFERENCE_OCC", "SLATER_EXPONENT", "P_SELFENERGY", "P_DKERNEL",
        "P_QKERNEL", "P_VCN", "P_RAD", "NSHELL", "ANG_SHELL", "PRINCIPAL_QUANTUM_NUMBER",
        "NUMBER_OF_PRIMITIVES",
    ],
    "crates/axtb/src/param/sto_data.rs": [
        "P_ALPHA1", "P_ALPHA2", "P_COEFF2", "P_ALPHA3", "P_COEFF3", "P_ALPHA4", "P_COEFF4",
        "P_ALPHA5", "P_COEFF5", "P_ALPHA6", "P_COEFF6", "P_ALPHA_6S", "P_COEFF_6S",
        "P_ALPHA_6P", "P_COEFF_6P",
    ],
    "crates/axtb/src/param/eeq_data.rs": ["EEQ_CHI", "EEQ_ETA", "EEQ_KCNCHI", "EEQ_RAD"],
    "crates/base/src/elements.rs": ["PAULING_EN", "COVALENT_RAD_2009_AA"],
    # the xtb 6.8.0 program's element tables (its conventions row)
    "crates/axtb/src/param/xtb_data.rs": [
        "XTB_COVALENT_RAD_D3", "XTB_ATOMIC_RAD", "XTB_PAULING_EN", "XTB_D4_RCOV", "XTB_D4_EN",
    ],
    "crates/d4/src/data.rs": [
        "CHEMICAL_HARDNESS", "EFFECTIVE_NUCLEAR_CHARGE", "R4_OVER_R2", "REFN", "REFQ_GFN2",
        "REFH_GFN2", "HCOUNT", "ASCALE", "REFCOVCN", "REFCN", "REFSYS", "ALPHAIW", "SSCALE",
        "SECAIW",
    ],
}

DECL = re.compile(r"pub\s+(?:const|static)\s+(\w+)\s*:\s*([^=]+)=\s*\[", re.S)


def strip_comments(text: str) -> str:
    return re.sub(r"//[^\n]*", "", text)


def extract(text: str, name: str):
    """The literal array `name` of a Rust source as a nested Python list of numbers."""
    for m in DECL.finditer(text):
        if m.group(1) != name:
            continue
        start = m.end() - 1
        depth = 0
        for i in range(start, len(text)):
            c = text[i]
            if c == "[":
                depth += 1
            elif c == "]":
                depth -= 1
                if depth == 0:
                    body = text[start:i + 1]
                    break
        else:
            raise ValueError(f"unterminated array {name}")
        rtype = m.group(2).strip()
        is_int = any(t in rtype for t in ("usize", "u8", "u32", "i32"))
        body = strip_comments(body)
        value = eval(body, {"__builtins__": {}}, NAMES)
        return value, is_int
    raise KeyError(name)


def shape(v):
    s = []
    while isinstance(v, list):
        s.append(len(v))
        v = v[0]
    return s


def flat(v):
    if isinstance(v, list):
        for x in v:
            yield from flat(x)
    else:
        yield v


def main() -> None:
    lines = [
        "// Generated by gen_params.py from the parameter arrays of axtb (LGPL-3.0-or-later);",
        "// do not edit. GFN2-xTB (JCTC 15, 1652 (2019)), STO-nG, EEQ-2019 and DFT-D4 tables.",
        "#pragma once",
        "",
        "namespace gfn2tab {",
        "",
    ]
    for rel, names in SOURCES.items():
        text = (REF / rel).read_text()
        lines.append(f"// ---- from {rel}")
        for name in names:
            value, is_int = extract(text, name)
            dims = shape(value)
            items = list(flat(value))
            ctype = "int" if is_int else "double"
            fmt = (lambda x: str(int(x))) if is_int else (lambda x: repr(float(x)))
            dim = "".join(f"[{d}]" for d in dims)
            lines.append(f"static const {ctype} {name}{dim} = {{")
            per = 6
            for k in range(0, len(items), per):
                lines.append("  " + ", ".join(fmt(x) for x in items[k:k + per]) + ",")
            lines.append("};")
        lines.append("")
    lines.append("}  // namespace gfn2tab")
    OUT.write_text("\n".join(lines) + "\n")
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
