import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    import json
    import numpy as np
    d = json.loads((ROOT / "tests" / "golden" / "reference_tables.json").read_text())
    h = lambda v: np.array([float.fromhex(x) for x in v])
    return {
        "Ke": h(d["Ke_nu0.3_cell1"]).reshape(24, 24, order="F"),
        "RI2": h(d["RI2"]).reshape(27, 8, order="F"),
        "RI4": h(d["RI4"]).reshape(125, 8, order="F"),
        "SUB2": np.array(d["SUB2"]),
        "SUB4": np.array(d["SUB4"]),
    }
