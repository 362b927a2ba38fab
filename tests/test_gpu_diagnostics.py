"""Solve-loop diagnostics, end-of-run files and restart of the GPU path.

* CFL (NavierStokes2DComputeCFL.c:19-56) and the residual norm of a step
  (TimePostStep.c:36-54) against the CPU oracle, step by step.
* The TimePrintStep lines (TimePrintStep.c:25-37) the drop-in CLI prints,
  and its errors.dat / conservation.dat / function_counts.dat
  (SimulationWriteErrors.c:65-80, CalculateError.c:30-120), against the
  reference binary on the same deck.
* Restart (restart_iter, ReadInputs.c:478-482, TimeInitialize.c:51,
  InitializeSolvers.c:240-245) from an intermediate op file converted to
  initial.inp as Extras/BinaryOPToInitialSolution.c does, against the
  reference's uninterrupted run and the reference's own restart.
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from oracle import oracle
from piafs_b200 import Simulation, deck
from test_gpu_parity import assert_close

pytestmark = pytest.mark.gpu
CLI = os.path.join(ROOT, "piafs_b200", "bin", "piafs-gpu")
REF = os.path.join(ROOT, "oracle", "_ref", "PIAFS")


def need(path):
    if not os.access(path, os.X_OK):
        pytest.skip(f"{os.path.basename(path)} not built")
    return path


def copy_deck(name, dst, **solver):
    shutil.copytree(os.path.join(GOLDEN, name), dst,
                    ignore=shutil.ignore_patterns("ref_final.bin", "ref_op_species_*"))
    p = os.path.join(dst, "solver.inp")
    txt = open(p).read()
    for k, v in solver.items():
        if re.search(rf"^\s*{k}\s", txt, re.M):
            txt = re.sub(rf"^(\s*){k}\s+\S+", rf"\g<1>{k} {v}", txt, flags=re.M)
        else:
            txt = txt.replace("end", f"  {k} {v}\nend", 1)
    open(p, "w").write(txt)
    return dst


def run(exe, d):
    r = subprocess.run([exe], cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def test_cfl_and_residual_norm_against_the_oracle(tmp_path):
    """The CFL is a maximum over interior points (no cancellation: 1e-12);
    the norm is an RMS of the step's change u_new - u_old, a difference of
    nearly equal states, so it carries the states' agreement (1e-14 of |u|)
    divided by |u_new - u_old| / |u| (about 1e-5 here): 1e-8."""
    d = copy_deck("ns2d_chem_crweno5_llf_64x48", str(tmp_path / "d"))
    case = oracle.load(d)
    u, t = case.u0.copy(), 0.0
    npts = case.dims[0] * case.dims[1]
    with Simulation(d) as sim:
        dt = sim.info["dt"]
        for k in range(10):
            c_gpu = sim.cfl()
            c_ref = case.cfl(u)
            assert abs(c_gpu - c_ref) <= 1e-12 * c_ref, (k, c_gpu, c_ref)
            n_gpu = sim.time_rk_norm(1)
            u1 = case.run(nsteps=1, u=u, t0=t)
            n_ref = np.sqrt(((case.interior(u1) - case.interior(u)) ** 2).sum() / npts)
            assert abs(n_gpu - n_ref) <= 1e-8 * n_ref, (k, n_gpu, n_ref)
            u, t = u1, t + dt


def printed(out):
    return re.findall(r"iter=\s*(\d+)\s+t=(\S+)\s+CFL=(\S+)\s+norm=(\S+)", out)


def dat(path):
    return [float(x) for x in open(path).read().split()]


def test_cli_prints_and_writes_what_the_reference_does(tmp_path):
    name = "ns2d_chem_crweno5_llf_64x48"
    dg = copy_deck(name, str(tmp_path / "gpu"), screen_op_iter=5)
    dc = copy_deck(name, str(tmp_path / "cpu"), screen_op_iter=5)
    # an exact solution file (here the initial state) makes both compute the
    # L1 / L2 / Linf error of the final solution against it
    for d in (dg, dc):
        shutil.copy(os.path.join(d, "initial.inp"), os.path.join(d, "exact.inp"))
    pg = printed(run(need(CLI), dg))
    pc = printed(run(need(REF), dc))
    assert len(pg) == len(pc) == 12 and pg == pc
    assert dat(os.path.join(dg, "function_counts.dat")) == dat(os.path.join(dc, "function_counts.dat"))
    assert dat(os.path.join(dg, "conservation.dat")) == dat(os.path.join(dc, "conservation.dat"))
    eg, ec = dat(os.path.join(dg, "errors.dat")), dat(os.path.join(dc, "errors.dat"))
    # grid, processes and dt exactly; errors to rounding; runtimes differ
    assert eg[:5] == ec[:5]
    assert np.allclose(eg[5:8], ec[5:8], rtol=1e-10, atol=0) and min(ec[5:8]) > 0


def test_restart_from_an_intermediate_output(tmp_path):
    """Run to step 30 of 60 writing op files, turn op_00001.bin into
    initial.inp and restart with restart_iter 30: the GPU's final solution
    matches the reference's uninterrupted run and the reference's restart.
    A restart writes no file at its first iteration and fast-forwards the
    file index by the outputs of the steps it skips, not counting the initial
    one (InitializeSolvers.c:240-245, Solve.cpp:57-67), so both restarts
    name their final solution op_00001.bin."""
    name = "ns2d_chem_crweno5_llf_64x48"
    full = copy_deck(name, str(tmp_path / "full"), file_op_iter=30)
    run(need(REF), full)
    assert os.path.exists(os.path.join(full, "op_00002.bin"))
    mid = deck.read_op(os.path.join(full, "op_00001.bin"))
    restarts = {}
    for who in ("gpu", "ref"):
        d = copy_deck(name, str(tmp_path / f"restart_{who}"), file_op_iter=30, restart_iter=30)
        deck.write_array_binary(os.path.join(d, "initial.inp"), mid.grid, mid.u)
        if who == "gpu":
            with Simulation(d) as sim:
                assert sim.info["iter"] == 30 and abs(sim.info["t"] - 30 * sim.info["dt"]) < 1e-15
                sim.solve(d)
        else:
            run(need(REF), d)
        outs = sorted(f for f in os.listdir(d) if re.fullmatch(r"op_\d{5}\.bin", f))
        assert outs == ["op_00001.bin"], outs
        restarts[who] = deck.read_op(os.path.join(d, "op_00001.bin")).u
    ref_full = deck.read_op(os.path.join(full, "op_00002.bin")).u
    assert_close(restarts["gpu"], ref_full, what="restart vs uninterrupted")
    assert_close(restarts["gpu"], restarts["ref"], what="restart vs the reference's restart")
