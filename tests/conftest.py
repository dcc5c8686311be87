import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import __graft_entry__ as ge  # noqa: E402

ge.load()

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the engine through its C ABI")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN_DIR, "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def svc():
    from altopir_b200 import service
    return service


@pytest.fixture(scope="session")
def eng():
    from altopir_b200 import engine
    return engine


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected on a machine without CUDA")
    from altopir_b200 import engine
    engine.init()
    return True


def sha(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="session")
def client_mod():
    from altopir_b200 import client
    return client


@pytest.fixture(scope="session")
def scheme_state(oracle, svc):
    """Engine state of the scheme itself (hint, InspiRING precomputation, prefixes) for a 4 MiB database of 2048
    synthetic records x 2048 bytes, built by the oracle's numpy restatement: requests of the client decrypt over it."""
    from oracle.scheme import SchemeState
    p = svc.params(2048, 2048)
    return SchemeState(p, oracle.synthetic_db_col(p.rows, 0, p.record_bytes), oracle)
