"""Shared test configuration.

Tests marked ``gpu`` need an sm_100 GPU and the built engine library; everything
else runs on the CPU.  The oracle (``oracle/``) is the checker: the C
restatement and, where built, the reference CPU engine in ``oracle/_ref``.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU and the built engine")


def load_golden(name):
    with np.load(GOLDEN / f"{name}.npz", allow_pickle=False) as f:
        return {k: f[k] for k in f.files}


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def reference_engine():
    import oracle
    ref = oracle.reference()
    if ref is None:
        pytest.skip("reference CPU engine not built (make -C oracle)")
    return ref
