"""Boundary zones, fourth-order viscous derivatives and the fifth-order upwind
scheme beyond the benchmark configurations.

Whole runs of these options are pinned by the golden decks the reference
itself produced (test_gpu_parity runs every golden deck); here the single
operators the goldens cannot isolate are checked against short numpy
restatements of the reference (BCReflect.c, BCDirichlet.c,
FirstDerivativeFourthOrder.c), and the batched engine against the same
goldens and against single runs.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from piafs_b200 import Batch, PiafsError, Simulation, cases, deck

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

BIG = 1e99
Z = deck.BoundaryZone


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


def rel_l2(got, ref):
    """Per-variable relative L2 (CompareSolutions.c:812-906), absolute where
    the reference norm vanishes."""
    num = np.sqrt(((got - ref) ** 2).sum(axis=0))
    den = np.sqrt((ref ** 2).sum(axis=0))
    return np.where(den > 1e-15, num / np.maximum(den, 1e-300), num)


def slab(zone, N, g):
    """Ghost indices of a zone along its dimension and their mirrored
    interior sources (BCReflect.c:38-41, BCDirichlet.c: the same slab)."""
    b = np.arange(g)
    if zone.face == 1:
        return -g + b, g - 1 - b
    return N[zone.dim] + b, N[zone.dim] - b - 1


def test_reflect_and_dirichlet_ghosts(tmp_path):
    """ApplyBoundaryConditions with reflect and Dirichlet zones: each zone
    writes its ghost slab, in the deck's order, the other dimension's
    extent by FindInterval over the interior points."""
    d = str(tmp_path / "rd")
    dval = [1.5, -0.25, 0.5, 3.0]
    zones = [Z("reflect", 0, 1, [0, 0, -BIG, BIG]), Z("dirichlet", 0, -1, [0, 0, -BIG, BIG], values=dval),
             Z("reflect", 1, 1, [0.3, BIG, 0, 0]), Z("reflect", 1, -1, [-BIG, BIG, 0, 0])]
    cases.ns2d_channel(d, zones, N=20, NY=12, n_iter=1, par="2")
    g, N = 3, (20, 12)
    x = (np.arange(20) + 0.5) / 20
    u = np.random.default_rng(5).uniform(0.5, 2.0, (N[1] + 2 * g, N[0] + 2 * g, 4))
    want = u.copy()
    for z in zones:
        gi, src = slab(z, N, g)
        if z.dim == 0:
            rows = np.arange(N[1]) + g
            for k in range(g):
                want[rows, gi[k] + g] = dval if z.bctype == "dirichlet" else -1.0 * want[rows, src[k] + g]
        else:
            cols = np.nonzero((x >= z.extent[0]) & (x <= z.extent[1]))[0] + g
            for k in range(g):
                want[gi[k] + g, cols] = -1.0 * want[src[k] + g, cols]
    with Simulation(d) as sim:
        t = dev(u.reshape(-1))
        sim.ApplyBoundaryConditions(t)
        got = host(t).reshape(u.shape)
    assert np.array_equal(got, want)


def d4_line(f, N, g):
    """FirstDerivativeFourthOrderCentral (FirstDerivativeFourthOrder.c:68-127)
    along the last axis of f (ghosted, N interior points, g ghosts)."""
    Df = np.zeros_like(f)
    c = 1.0 / 12.0
    for k in range(N + 2 * g):
        i = k - g
        if i == -g:
            Df[..., k] = (-25 * f[..., k] + 48 * f[..., k + 1] - 36 * f[..., k + 2] + 16 * f[..., k + 3]
                          - 3 * f[..., k + 4]) * c
        elif i == -g + 1:
            Df[..., k] = (-3 * f[..., k - 1] - 10 * f[..., k] + 18 * f[..., k + 1] - 6 * f[..., k + 2]
                          + f[..., k + 3]) * c
        elif i == N + g - 2:
            Df[..., k] = (-f[..., k - 3] + 6 * f[..., k - 2] - 18 * f[..., k - 1] + 10 * f[..., k]
                          + 3 * f[..., k + 1]) * c
        elif i == N + g - 1:
            Df[..., k] = (3 * f[..., k - 4] - 16 * f[..., k - 3] + 36 * f[..., k - 2] - 48 * f[..., k - 1]
                          + 25 * f[..., k]) * c
        else:
            Df[..., k] = (f[..., k - 2] - 8 * f[..., k - 1] + 8 * f[..., k + 1] - f[..., k + 2]) * c
    return Df


@pytest.mark.parametrize("bias", [1, -1])
def test_first_derivative_fourth_order(tmp_path, bias):
    """FirstDerivativePar with par_space_scheme 4: the central stencil inside,
    the biased rows at the two outermost points, on the lines that are
    interior in the other dimension (the bias is not used)."""
    d = str(tmp_path / "p4")
    cases.ns2d_channel(d, [Z("extrapolate", k, f, [0, 0, -BIG, BIG] if k == 0 else [-BIG, BIG, 0, 0])
                           for k in (0, 1) for f in (1, -1)], N=24, NY=14, n_iter=1, par="4")
    g, N0, N1, nv = 3, 24, 14, 4
    f = np.random.default_rng(7).uniform(-1, 1, (N1 + 2 * g, N0 + 2 * g, nv))
    with Simulation(d) as sim:
        for dr in (0, 1):
            want = np.zeros_like(f)
            if dr == 0:
                want[g:g + N1] = np.moveaxis(d4_line(np.moveaxis(f[g:g + N1], 1, -1), N0, g), -1, 1)
            else:
                want[:, g:g + N0] = np.moveaxis(d4_line(np.moveaxis(f[:, g:g + N0], 0, -1), N1, g), -1, 0)
            t = dev(np.zeros(f.size))
            sim.FirstDerivativePar(t, dev(f.reshape(-1)), dr, bias, nv)
            got = host(t).reshape(f.shape)
            np.testing.assert_allclose(got, want, rtol=0, atol=1e-14)


FLOW_GOLDEN = ["ns2d_ambivalent_dirichlet_weno5_llf_40x32", "ns2d_chem_supersonic_jet_weno5_rf_24x32",
               "euler1d_weno5_roe_dirichlet_n128"]


def test_batch_flow_boundaries_match_the_reference():
    """Batched members with Dirichlet, subsonic ambivalent and supersonic
    inflow / outflow zones (ghosts computed on the fly in the stage tile)
    against the reference's own output."""
    with Batch() as b:
        ids = {name: b.add(os.path.join(GOLDEN, name)) for name in FLOW_GOLDEN}
        b.step(1000)
        for name, i in ids.items():
            got = b.solution(i)
            ref = deck.read_op(os.path.join(GOLDEN, name, "ref_final.bin")).u
            assert rel_l2(got, ref).max() <= 1e-12, name


def test_batch_upw5_walls_match_single_run(tmp_path):
    """A batched upw5 member with no-slip walls, a subsonic inflow and outflow
    matches the same deck run alone."""
    d = str(tmp_path / "upw5")
    zones = [Z("subsonic-inflow", 0, 1, [0, 0, -BIG, BIG], values=[1.0, 0.3, 0.0]),
             Z("subsonic-outflow", 0, -1, [0, 0, -BIG, BIG], values=[1 / 1.4]),
             Z("noslip-wall", 1, 1, [-BIG, BIG, 0, 0], [0.0, 0.0]),
             Z("noslip-wall", 1, -1, [-BIG, BIG, 0, 0], [0.05, 0.0])]
    cases.ns2d_channel(d, zones, N=40, NY=24, n_iter=30, scheme="upw5", par="2", op_file_format="none")
    with Simulation(d) as sim:
        sim.time_rk(30)
        alone = sim.solution()
    with Batch() as b:
        i = b.add(d)
        b.step(30)
        got = b.solution(i)
    nv = 4
    assert rel_l2(got.reshape(-1, nv), alone.reshape(-1, nv)).max() <= 1e-12


def test_batch_refuses_fourth_order_viscous_terms(tmp_path):
    d = str(tmp_path / "p4")
    cases.ns2d_channel(d, [Z("extrapolate", k, f, [0, 0, -BIG, BIG] if k == 0 else [-BIG, BIG, 0, 0])
                           for k in (0, 1) for f in (1, -1)], N=32, n_iter=2, par="4", op_file_format="none")
    with Batch() as b:
        with pytest.raises(PiafsError) as ex:
            b.add(d)
        assert ex.value.code == 3
