"""The passive variables' interface values packed for their upwinding
(uL - uR and fL + fR written by the CRWENO5 line solve, DevParams::pack_sp)
against the four separate interface arrays on the same deck: the same values
bit for bit, in FP64 and mixed precision, for the upwinding schemes that pack
(LLF, Roe, Rusanov; RF keeps the four arrays), on the transposed and on the
column-strided y pass.  The parity tests against the reference run the
packed form (it is the default wherever it applies).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from piafs_b200 import Simulation, cases

pytestmark = pytest.mark.gpu


def run(d, precision, packed, nsteps=10, extra=None):
    env = {"PIAFS_GPU_NO_PACKED_SPECIES": "0" if packed else "1"}
    env.update(extra or {})
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        with Simulation(d, precision=precision) as sim:
            sim.time_rk(nsteps)
            return sim.solution()
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v


def deck(tmp_path, name, upwinding):
    if upwinding is None:
        return os.path.join(GOLDEN, name)
    d = str(tmp_path / f"{name}_{upwinding}")
    cases.ns2d_photochem_beam(d, N=40, NY=36, n_iter=10, dt=0.4 / 2048, upwinding=upwinding, scheme="crweno5")
    return d


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name,upwinding", [("ns2d_chem_crweno5_llf_64x48", None), ("beam", "roe"),
                                            ("beam", "rusanov")])
def test_packed_species_equal_the_separate_arrays(tmp_path, name, upwinding, precision):
    d = deck(tmp_path, name, upwinding)
    packed = run(d, precision, True)
    sep = run(d, precision, False)
    assert np.isfinite(packed).all()
    assert np.array_equal(packed, sep), np.abs(packed - sep).max()


def test_packed_species_on_the_strided_y_pass():
    d = os.path.join(GOLDEN, "ns2d_chem_crweno5_llf_64x48")
    strided = {"PIAFS_GPU_NO_YTRANSPOSE": "1"}
    assert np.array_equal(run(d, "fp64", True, extra=strided), run(d, "fp64", False, extra=strided))
