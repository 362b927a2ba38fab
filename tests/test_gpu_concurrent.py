"""The y pass on its own stream, concurrent with the x pass (the default for
2D Navier-Stokes with a transposed y pass), against both passes on one
stream: the same kernels on the same inputs into separate buffers, so the
same solution bit for bit -- in FP64 and mixed precision, with the step
graphs and without them.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from piafs_b200 import Simulation

pytestmark = pytest.mark.gpu


def run(d, precision, concurrent, graph=True, nsteps=8):
    env = {"PIAFS_GPU_NO_CONCURRENT_Y": "0" if concurrent else "1", "PIAFS_GPU_NO_GRAPH": "0" if graph else "1"}
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


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("graph", [True, False])
def test_concurrent_y_pass_equals_one_stream(precision, graph):
    d = os.path.join(GOLDEN, "ns2d_chem_crweno5_llf_64x48")
    a = run(d, precision, True, graph)
    b = run(d, precision, False, graph)
    assert np.isfinite(a).all()
    assert np.array_equal(a, b)
