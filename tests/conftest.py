import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def golden_cases():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        return json.load(f)


def load_golden(case):
    with open(os.path.join(GOLDEN, case["json"])) as f:
        return json.load(f)


def case_id(case):
    return f"{case['name']}-k{case['k']}"


@pytest.fixture(scope="session")
def ctx():
    import cds_b200 as cds
    c = cds.Context(0)
    yield c
    c.close()
