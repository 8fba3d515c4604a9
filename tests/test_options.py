"""Option checks of the C ABI on the host (CPU: axtb_gpu_create validates before any device work).

Unknown conventions, mixers, solvation models, solvents and reference states are input errors
(crates/axtb/src/scf/mixing.rs:202-214, crates/solvation/src/lib.rs:255-272); xtb's solvent
aliases resolve in any case.
"""
import pytest

import axtb_b200 as A


@pytest.mark.parametrize("opts", [dict(conventions="xtb671"), dict(mixer="anderson2"),
                                  dict(solvation=("alpb", "vacuum")), dict(solvation=("cosmo", "water")),
                                  dict(solvation=("gbsa", "water", "standard")), dict(precision="fp32")])
def test_invalid_options_are_input_errors(opts):
    with pytest.raises((A.AxtbError, KeyError)) as e:
        A.Calculator([8, 1, 1], **opts)
    if isinstance(e.value, A.AxtbError):
        assert e.value.kind == "input"


@pytest.mark.parametrize("opts", [dict(conventions="tblite", mixer="DIIS"), dict(mixer="pulay"),
                                  dict(solvation=("alpb", "H2O")), dict(solvation=("gbsa", "Chloroform", "bar1M")),
                                  dict(solvation=("ALPB", "dichloromethane", "reference"))])
def test_valid_options_create(opts):
    A.Calculator([8, 1, 1], **opts).close()


@pytest.mark.parametrize("numbers,kw,kind", [
    ([8, 1, 1], dict(uhf=1), "input"),              # unpaired electrons of the wrong parity
    ([1], dict(charge=2.0), "input"),               # a negative electron count
    ([1, 1], dict(uhf=4), "input"),                 # more unpaired electrons than electrons
    ([8, 1, 1], dict(charge=0.5), "input"),         # fractional electron counts
    ([87], {}, "unsupported_element"),              # beyond GFN2-xTB's elements
    ([], {}, "input"),                              # no atoms
])
def test_molecule_checks(numbers, kw, kind):
    """crates/base/src/molecule.rs:35-99 and the electron count of crates/axtb/src/xtb.rs:1178-1212,
    checked when the handle is created."""
    with pytest.raises(A.AxtbError) as e:
        A.Calculator(numbers, **kw)
    assert e.value.kind == kind


def test_heaviest_element_is_accepted():
    A.Calculator([86]).close()
