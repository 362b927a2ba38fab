"""Mixed-precision path (FP32 inner arithmetic on FP64 state) against FP64.

The mixed path computes reconstruction weights and rows, upwind fluxes,
viscous stencils and the chemistry source in FP32, and keeps the conserved
state, the RK stage accumulation and the CRWENO5 tridiagonal solves in FP64.
Its error is stated against the FP64 GPU path on the same deck: relative L2
per conserved variable (CompareSolutions-style), bounded by MIXED_TOL; the
relative Linf is printed beside it.  Variables that carry no signal (RMS below
NOISE_FLOOR x the largest variable RMS) are held to the bound in absolute
terms scaled by that largest RMS, as in the FP64 parity tests.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden_cases
from piafs_b200 import Simulation, deck

pytestmark = pytest.mark.gpu
MIXED_TOL = 1e-5
NOISE_FLOOR = 1e-6


def mixed_error(got, ref):
    got = np.asarray(got).reshape(ref.shape)
    assert np.all(np.isfinite(got)), "non-finite values in the mixed run"
    rms = np.sqrt((ref * ref).mean(axis=0))
    scale = rms.max()
    l2, linf = [], []
    for v in range(ref.shape[1]):
        d = got[:, v] - ref[:, v]
        if rms[v] < NOISE_FLOOR * scale:
            l2.append(np.sqrt((d * d).mean()) / scale)
            linf.append(np.abs(d).max() / scale)
        else:
            l2.append(np.sqrt((d * d).sum() / (ref[:, v] ** 2).sum()))
            linf.append(np.abs(d).max() / np.abs(ref[:, v]).max())
    return np.array(l2), np.array(linf)


def run(d, precision, steps=None):
    with Simulation(d, precision=precision) as sim:
        n = sim.info["n_iter"] if steps is None else steps
        sim.time_rk(n)
        return sim.solution(), sim.info["nvars"]


@pytest.mark.parametrize("name", golden_cases(components_only=True))
def test_mixed_tracks_fp64(name):
    d = os.path.join(GOLDEN, name)
    ref, nv = run(d, "fp64")
    got, _ = run(d, "mixed")
    l2, linf = mixed_error(got.reshape(-1, nv), ref.reshape(-1, nv))
    print(f"{name}: mixed vs FP64 rel L2 max {l2.max():.2e}, rel Linf max {linf.max():.2e}")
    assert l2.max() <= MIXED_TOL, f"rel L2 per var {[f'{x:.1e}' for x in l2]}"


def test_mixed_against_reference_output():
    """The mixed run of the 2D photochemical golden deck also stays within the
    bound of the reference's own FP64 output."""
    name = "ns2d_chem_crweno5_llf_64x48"
    d = os.path.join(GOLDEN, name)
    got, nv = run(d, "mixed")
    ref = deck.read_op(os.path.join(d, "ref_final.bin")).u
    l2, _ = mixed_error(got.reshape(-1, nv), ref.reshape(-1, nv))
    assert l2.max() <= MIXED_TOL


def test_mixed_operator_entry_points_stay_fp64():
    """InterpolateInterfacesHyp of a mixed simulation is the FP64 operator."""
    torch = pytest.importorskip("torch")
    d = os.path.join(GOLDEN, "ns2d_chem_crweno5_llf_64x48")
    out = []
    for prec in ("fp64", "mixed"):
        with Simulation(d, precision=prec) as sim:
            u = torch.from_numpy(sim.state()).cuda()
            f = torch.zeros_like(u)
            sim.FFunction(f, u, 0)
            ni = sim.info["ninterfaces"][0] * sim.info["nvars"]
            fi = torch.zeros(ni, dtype=torch.float64, device="cuda")
            sim.InterpolateInterfacesHyp(fi, f, u, 1, 0, 0)
            out.append(fi.cpu().numpy())
    assert np.array_equal(out[0], out[1])


def test_mixed_full_size_2048(tmp_path):
    """The 2048^2 photochemical workload, 6 SSPRK3 steps through the heating
    pulse: the mixed path stays within the bound of FP64."""
    from piafs_b200 import cases
    d = str(tmp_path / "beam")
    cases.ns2d_photochem_beam(d, N=2048, n_iter=6, scheme="crweno5", op_file_format="none", dt=0.4 / 2048)
    ref, nv = run(d, "fp64")
    got, _ = run(d, "mixed")
    l2, linf = mixed_error(got.reshape(-1, nv), ref.reshape(-1, nv))
    print(f"2048^2: mixed vs FP64 rel L2 max {l2.max():.2e}, rel Linf max {linf.max():.2e}")
    assert l2.max() <= MIXED_TOL
