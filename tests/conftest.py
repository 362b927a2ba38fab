import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def interp_type(d):
    """hyp_interp_type of a deck directory (the reference's default when absent)."""
    for line in open(os.path.join(d, "solver.inp")):
        parts = line.split()
        if len(parts) >= 2 and parts[0] == "hyp_interp_type":
            return parts[1]
    return "characteristic"


def has_sponge(d):
    return "sponge" in open(os.path.join(d, "boundary.inp")).read().split()


def golden_cases(components_only=False, no_sponge=False):
    """Golden fixture names; components_only leaves out the decks that
    interpolate characteristic variables (the CPU oracle and the mixed
    precision path restate component-wise interpolation only), no_sponge the
    decks with sponge zones (not restated by the CPU oracle)."""
    names = sorted(d for d in os.listdir(GOLDEN) if os.path.isfile(os.path.join(GOLDEN, d, "ref_final.bin")))
    if components_only:
        names = [n for n in names if interp_type(os.path.join(GOLDEN, n)) == "components"]
    if no_sponge:
        names = [n for n in names if not has_sponge(os.path.join(GOLDEN, n))]
    return names


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
