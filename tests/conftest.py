import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))

GOLDEN = os.path.join(REPO, "tests", "golden")
C100K_1P = os.path.join(REPO, "oracle", "_ref", "c100k")
REF_BIN = os.path.join(REPO, "oracle", "_ref", "gip_ref_cpu")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: a full-size configuration check (minutes)")


def have_c100k() -> bool:
    return os.path.isdir(os.path.join(C100K_1P, "InputFiles"))


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def c100k_case():
    if not have_c100k():
        pytest.skip("merged C100K set not built (tests/golden/make_goldens.py)")
    from gip_b200 import formats
    return formats.load_case(C100K_1P, "C100K", 1, 0)


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from gip_b200 import _lib
    _lib.load()
    return torch.device("cuda:0")


def golden_lines(name: str):
    with open(os.path.join(GOLDEN, name)) as f:
        return [ln.rstrip("\n") for ln in f if ln.strip()]


def rel_err(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))
