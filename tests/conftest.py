import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden" / "golden.npz"
GROUPS = ("C2", "C3", "C4", "C6", "D2", "D3", "D4", "D6", "T", "O", "I")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the engine's kernels")
    config.addinivalue_line("markers", "slow: long-running GPU parity case")


@pytest.fixture(scope="session")
def golden():
    with np.load(GOLDEN) as data:
        return {k: data[k] for k in data.files}


@pytest.fixture(scope="session")
def ops64(golden):
    """FP64 operator tables (the reference's published group tables)."""
    return {g: golden[f"ops_{g}"] for g in GROUPS}


@pytest.fixture(scope="session")
def ops32(golden):
    """The float32 tables the reference uploads, as FP64 values."""
    return {g: golden[f"ops_{g}"].astype(np.float32).astype(np.float64) for g in GROUPS}


@pytest.fixture(scope="session")
def engine():
    """The built engine package (GPU tests); fails loudly when the library is missing."""
    import zxtalori_b200 as zo

    if not zo.library_path().is_file():
        pytest.fail(f"engine library missing: {zo.library_path()}")
    return zo
