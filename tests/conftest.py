import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "final-single-block-_b200"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU run")


def pytest_sessionfinish(session, exitstatus):
    out = os.environ.get("LH_PARITY_OUT")
    if not out:
        return
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import json

    from helpers import PARITY_RECORD
    if PARITY_RECORD:
        with open(out, "w") as f:
            json.dump(PARITY_RECORD, f, indent=1)


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN
