"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; the rest run on CPU."""
from __future__ import annotations

import glob
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

GOLDEN = os.path.join(ROOT, "tests", "golden")
# every device wait in a test is bounded tightly, so a wait bug surfaces as
# MCE_ERR_TIMEOUT instead of a long stall
TEST_SPIN = 1 << 22


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run on the B200 box)")


def golden_fixtures():
    out = []
    for path in sorted(glob.glob(os.path.join(GOLDEN, "*.json"))):
        with open(path) as f:
            out.append(json.load(f))
    return out


def edges_uv(fx):
    e = np.asarray(fx["edges"], dtype=np.uint64).reshape(-1, 2)
    return e[:, 0].astype(np.uint32), e[:, 1].astype(np.uint32)


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def engine():
    import rdmce_b200

    return rdmce_b200


@pytest.fixture(scope="session")
def gpu(engine):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return engine


def opts(engine, **kw):
    kw.setdefault("spin_limit", TEST_SPIN)
    return engine.options(**kw)
