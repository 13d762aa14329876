import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN_DIR, "golden.json")) as f:
        return json.load(f)["fixtures"]


@pytest.fixture(scope="session")
def fixtures():
    return dict(np.load(os.path.join(GOLDEN_DIR, "fixtures.npz")))


def edge_fixture_names(golden_dict, fixtures_dict):
    return [n for n in golden_dict if n + "_src" in fixtures_dict]


def load_golden():
    with open(os.path.join(GOLDEN_DIR, "golden.json")) as f:
        return json.load(f)["fixtures"]


def load_golden_large():
    """Counts of the full-size benchmark graphs pinned on the CPU by
    tests/golden/make_golden_large.py (both oracle counters, and the
    reference's own binary where recorded)."""
    with open(os.path.join(GOLDEN_DIR, "golden.json")) as f:
        return json.load(f).get("large", {})


def load_fixtures():
    return dict(np.load(os.path.join(GOLDEN_DIR, "fixtures.npz")))
