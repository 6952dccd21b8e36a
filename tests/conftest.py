import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a kernels")


def _ensure_built():
    from matrix_format_performance_b200 import build as b
    b.build()
    import oracle
    if not oracle.oracle.ORACLE_SO.exists():
        oracle.build(ref=False)


_ensure_built()


def golden_cases():
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load_golden(name):
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import load_oracle
    return load_oracle()


@pytest.fixture(scope="session")
def ref_lib():
    from oracle import load_ref
    return load_ref()
