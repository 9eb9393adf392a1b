import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / "thesis-source-code_b200", ROOT / "oracle", ROOT / "tests" / "golden"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def ctx():
    import vtib200 as V
    c = V.Context(0)
    yield c
    c.close()


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def load_golden(name):
    f = ROOT / "tests" / "golden" / f"{name}.npz"
    if not f.exists():
        pytest.fail(f"golden fixture {f.name} missing (generate with tests/golden/make_golden.py)")
    return dict(np.load(f))
