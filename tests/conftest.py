import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a engine")


@pytest.fixture(scope="session")
def golden():
    import json

    data = json.loads((ROOT / "tests" / "golden" / "reference_matrix.json").read_text())
    return {c["id"]: c for c in data["cases"]}


@pytest.fixture(scope="session")
def engine():
    """The built engine; GPU tests fail (not skip) when the library is missing."""
    from axtb_b200 import build

    build.build()
    import axtb_b200

    return axtb_b200
