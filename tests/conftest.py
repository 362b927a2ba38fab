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


def solver_key(d, key, default):
    for line in open(os.path.join(d, "solver.inp")):
        parts = line.split()
        if len(parts) >= 2 and parts[0] == key:
            return parts[1]
    return default


# what the CPU oracle restates: the benchmark configurations' schemes and
# boundaries (component-wise WENO5 / CRWENO5, second-order viscous terms,
# periodic / extrapolate / slip-wall zones)
ORACLE_BOUNDARIES = {"periodic", "extrapolate", "slip-wall"}


def in_oracle_scope(d):
    toks = open(os.path.join(d, "boundary.inp")).read().split()
    types = {t for t in toks if t[0].isalpha()}
    return (types <= ORACLE_BOUNDARIES and interp_type(d) == "components"
            and solver_key(d, "hyp_space_scheme", "1") in ("weno5", "crweno5")
            and solver_key(d, "par_space_scheme", "2") == "2")


def golden_cases(components_only=False, oracle_scope=False):
    """Golden fixture names; components_only leaves out the decks that
    interpolate characteristic variables (the mixed precision path restates
    component-wise interpolation only), oracle_scope the decks with options
    the CPU oracle does not restate (sponge, wall, inflow and outflow zones,
    fourth-order viscous terms, upw5; the reference's own output pins those)."""
    names = sorted(d for d in os.listdir(GOLDEN) if os.path.isfile(os.path.join(GOLDEN, d, "ref_final.bin")))
    if components_only:
        names = [n for n in names if interp_type(os.path.join(GOLDEN, n)) == "components"]
    if oracle_scope:
        names = [n for n in names if in_oracle_scope(os.path.join(GOLDEN, n))]
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
