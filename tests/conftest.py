import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def golden_cases():
    return sorted(d for d in os.listdir(GOLDEN) if os.path.isfile(os.path.join(GOLDEN, d, "ref_final.bin")))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture
def deck_copy(tmp_path):
    """Copy a golden deck (without its reference output) into a temp dir."""
    import shutil

    def _copy(name):
        d = tmp_path / name
        shutil.copytree(os.path.join(GOLDEN, name), d, ignore=shutil.ignore_patterns("ref_final.bin"))
        return str(d)

    return _copy
