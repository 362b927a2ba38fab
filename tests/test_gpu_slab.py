"""A 2D grid decomposed into row slabs (include/piafs_gpu.h piafs_gpu_slab_*,
piafs_b200/slab.py) against the same grid undecomposed, on one GPU: every
slab of the grid in one process (LocalSlabs), the exchanges as device
copies.  The decomposed solution must equal the undecomposed one bit for
bit: every value is formed by the same kernels from the same operands (the
y lines are solved whole on their column slab; the y term of the divergence
is rounded on its own and the x term's product fused onto it, on both
paths).
"""
import os
import shutil

import numpy as np
import pytest

from conftest import GOLDEN
from piafs_b200 import PiafsError, Simulation
from piafs_b200.slab import LocalSlabs

pytestmark = pytest.mark.gpu
NSTEPS = 5


def copy_deck(name, dst):
    shutil.copytree(os.path.join(GOLDEN, name), dst,
                    ignore=shutil.ignore_patterns("ref_final.bin", "ref_op_species_*"))
    return dst


def periodic_in_y(d):
    """The deck with its y faces periodic too (no golden deck is)."""
    with open(os.path.join(d, "boundary.inp"), "w") as f:
        f.write("4\n")
        f.write("periodic 0  1 0 0 -1e+99 1e+99\nperiodic 0 -1 0 0 -1e+99 1e+99\n")
        f.write("periodic 1  1 -1e+99 1e+99 0 0\nperiodic 1 -1 -1e+99 1e+99 0 0\n")
    return d


def whole_and_slabs(d, nranks, precision="fp64"):
    with Simulation(d, precision=precision) as sim:
        sim.time_rk(NSTEPS)
        ref = sim.solution()
    with LocalSlabs(d, nranks, precision=precision) as sl:
        sl.step(NSTEPS)
        got = sl.solution()
    return got, ref


@pytest.mark.parametrize("name,nranks", [
    ("ns2d_chem_crweno5_llf_64x48", 2), ("ns2d_chem_crweno5_llf_64x48", 4),
    ("ns2d_shear_weno5_roe_re200_40x32", 2), ("ns2d_shear_weno5_roe_re200_40x32", 4),
    ("ns2d_chem_supersonic_jet_weno5_rf_24x32", 4), ("ns2d_shear_crweno5_rusanov_inviscid_32x36", 4),
    ("ns2d_ambivalent_dirichlet_weno5_llf_40x32", 2), ("ns2d_chem_crweno5_rf_borges_32x32", 2),
])
def test_slabs_equal_the_whole_grid(tmp_path, name, nranks):
    d = copy_deck(name, str(tmp_path / name))
    got, ref = whole_and_slabs(d, nranks)
    assert got.shape == ref.shape and np.isfinite(ref).all()
    assert np.array_equal(got, ref), np.abs(got - ref).max()


@pytest.mark.parametrize("nranks", [2, 4])
def test_slabs_periodic_in_y(tmp_path, nranks):
    d = periodic_in_y(copy_deck("ns2d_shear_crweno5_llf_re200_48x40", str(tmp_path / "d")))
    got, ref = whole_and_slabs(d, nranks)
    assert np.array_equal(got, ref), np.abs(got - ref).max()


def test_slabs_mixed_precision(tmp_path):
    d = copy_deck("ns2d_chem_crweno5_llf_64x48", str(tmp_path / "d"))
    got, ref = whole_and_slabs(d, 2, precision="mixed")
    assert np.array_equal(got, ref), np.abs(got - ref).max()


@pytest.mark.parametrize("name,nranks,what", [
    ("ns2d_shear_weno5_llf_sponge_40x32", 2, "sponge"),
    ("ns2d_shear_crweno5char_llf_re200_40x32", 2, "characteristic"),
    ("ns2d_flatplate_subsonic_weno5_par4_48x24", 2, "par_space_scheme 4"),
    ("ns2d_chem_crweno5_llf_64x48", 5, "multiples"),
    ("ns2d_chem_weno5_llf_48x40", 2, "mixed precision"),
])
def test_slabs_refuse_what_they_do_not_cover(tmp_path, name, nranks, what):
    d = copy_deck(name, str(tmp_path / name))
    with pytest.raises(PiafsError, match=what):
        LocalSlabs(d, nranks, precision="mixed" if what == "mixed precision" else "fp64")


def _slab_rank(rank, world, port, d, out):
    """One rank of a decomposed run as its own process (gloo, so the
    exchanges go through host copies; both ranks share the one GPU, and no
    kernel of one waits on the other's)."""
    import torch
    import torch.distributed as dist
    from piafs_b200.slab import SlabSimulation
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        sim = SlabSimulation(d)
        u0 = sim.state()
        sim.step(2)
        sim.set_state(u0, 0.0)                 # back to the start: the same run again
        sim.step(NSTEPS - 1)
        norm = sim.step(1, norm=True)
        cfl = sim.cfl()
        sol = sim.gather_solution()
        sim.close()
        if rank == 0:
            np.save(out, sol)
            np.save(out + ".diag.npy", np.array([norm, cfl]))
    finally:
        dist.destroy_process_group()


def test_slabs_as_processes_over_gloo(tmp_path):
    import socket
    import torch.multiprocessing as mp
    d = copy_deck("ns2d_chem_crweno5_llf_64x48", str(tmp_path / "d"))
    with Simulation(d) as sim:
        sim.time_rk(NSTEPS - 1)
        norm_ref = sim.time_rk_norm(1)
        cfl_ref = sim.cfl()
        ref = sim.solution()
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    out = str(tmp_path / "sol.npy")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_slab_rank, args=(r, 2, port, d, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    assert np.array_equal(np.load(out), ref)
    norm, cfl = np.load(out + ".diag.npy")
    assert abs(norm - norm_ref) <= 1e-12 * norm_ref and abs(cfl - cfl_ref) <= 1e-14 * cfl_ref
