"""The passive variables' fused path (k_crw_species: reconstruction,
upwinding with the flow's speed and the flux difference in one kernel per
direction) against the separate upwind kernel on the same deck: the same
values bit for bit, in FP64 and mixed precision, for every upwinding scheme
(the species modes of Roe / Rusanov, LLF and RF).  The parity tests against
the reference run the fused path (it is the default wherever it applies).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from piafs_b200 import Simulation, cases

pytestmark = pytest.mark.gpu


def run(d, precision, fused, nsteps=10):
    old = os.environ.get("PIAFS_GPU_NO_FUSED_SPECIES")
    os.environ["PIAFS_GPU_NO_FUSED_SPECIES"] = "0" if fused else "1"
    try:
        with Simulation(d, precision=precision) as sim:
            per_step = sim.info["launches_per_step"]
            sim.time_rk(nsteps)
            return sim.solution(), per_step
    finally:
        if old is None:
            del os.environ["PIAFS_GPU_NO_FUSED_SPECIES"]
        else:
            os.environ["PIAFS_GPU_NO_FUSED_SPECIES"] = old


def deck(tmp_path, name, upwinding):
    if upwinding is None:
        return os.path.join(GOLDEN, name)
    d = str(tmp_path / f"{name}_{upwinding}")
    cases.ns2d_photochem_beam(d, N=40, NY=36, n_iter=10, dt=0.4 / 2048, upwinding=upwinding, scheme="crweno5")
    return d


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name,upwinding", [("ns2d_chem_crweno5_llf_64x48", None),
                                            ("ns2d_chem_crweno5_rf_borges_32x32", None),
                                            ("beam", "roe"), ("beam", "rusanov"), ("beam", "rf-char")])
def test_fused_species_equal_the_separate_upwind_kernel(tmp_path, name, upwinding, precision):
    d = deck(tmp_path, name, upwinding)
    fused, n_fused = run(d, precision, True)
    sep, n_sep = run(d, precision, False)
    assert n_fused == n_sep + 4 * 3     # speed + species kernels of two directions, three stages
    assert np.isfinite(fused).all()
    assert np.array_equal(fused, sep), np.abs(fused - sep).max()
