"""Parity at the benchmark's own scale.

The 2D photochemical Navier-Stokes workload (CRWENO5 on components, LLF,
SSPRK3, second-order viscous terms, periodic x / slip-wall y, dt = 0.4 / N)
written by the same generator the benchmark uses, run by the reference CPU
binary (llnl/piafs compiled from its own sources by oracle/Makefile,
oracle/_ref/PIAFS_omp on all host threads) and by the GPU path on the same
deck; the reference's final op file is the expected solution.  Tolerance:
relative L2 per conserved variable <= 1e-12 (CompareSolutions-style,
Extras/CompareSolutions.c:812-906), with the variables that hold no signal
yet (RMS below 1e-6 of the largest, e.g. the momenta a few steps after a
quiescent start, whose values are differences of O(1) pressures) held to
1e-12 of the state scale in absolute terms, as in tests/test_gpu_parity.py.

The mixed-precision path (FP32 reconstruction rows, weights, fluxes,
viscous and source terms on FP64 state, FP64 line solves) is held to the FP64
GPU path at 4096^2, the configuration its throughput is quoted on, within
1e-5 relative L2 per variable with signal; the Linf error is reported.
"""
import os
import subprocess
import time

import numpy as np
import pytest

from conftest import ROOT
from piafs_b200 import Simulation, cases, deck

pytestmark = pytest.mark.gpu
TOL = 1e-12
NOISE_FLOOR = 1e-6
MIXED_TOL = 1e-5


def reference_binary():
    for b in ("PIAFS_omp", "PIAFS"):
        p = os.path.join(ROOT, "oracle", "_ref", b)
        if os.access(p, os.X_OK):
            return p
    return None


def per_variable_error(got, ref):
    """Worst per-variable error: relative L2 where a variable holds signal,
    absolute RMS over the state scale where it does not."""
    norms = deck.rel_norms(got, ref)
    rms = np.sqrt((ref * ref).mean(axis=0))
    scale = rms.max()
    errs = []
    for v, n in enumerate(norms):
        if rms[v] < NOISE_FLOOR * scale:
            errs.append(float(np.sqrt(((got[:, v] - ref[:, v]) ** 2).mean()) / scale))
        else:
            errs.append(float(n[1]))
    return errs


@pytest.mark.parametrize("N,steps", [(512, 10), (2048, 2)])
def test_benchmark_workload_matches_the_reference_binary(tmp_path, N, steps):
    binary = reference_binary()
    if binary is None:
        pytest.skip("reference binary not built (make -C oracle)")
    d = str(tmp_path / f"bench_{N}")
    cases.ns2d_photochem_beam(d, N=N, n_iter=steps, dt=0.4 / N, op_file_format="binary")
    threads = len(os.sched_getaffinity(0))
    t0 = time.perf_counter()
    subprocess.run([binary], cwd=d, env=dict(os.environ, OMP_NUM_THREADS=str(threads)), check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    t_ref = time.perf_counter() - t0
    ref = deck.read_op(os.path.join(d, deck.op_filename(1))).u
    with Simulation(d) as sim:
        sim.time_rk(steps)
        got = sim.solution()
        assert sim.info["singular"] == 0
    assert np.all(np.isfinite(got))
    errs = per_variable_error(got, ref)
    print(f"{N}^2, {steps} steps: reference {t_ref:.1f} s on {threads} threads; "
          f"worst per-variable error {max(errs):.2e}")
    assert max(errs) <= TOL, f"per-variable errors {[f'{e:.2e}' for e in errs]}"


def test_mixed_precision_4096_against_fp64(tmp_path):
    d = str(tmp_path / "mixed_4096")
    N, steps = 4096, 4
    cases.ns2d_photochem_beam(d, N=N, n_iter=steps, dt=0.4 / N, op_file_format="none")
    with Simulation(d, precision="fp64") as sim:
        sim.time_rk(steps)
        ref = sim.solution()
    with Simulation(d, precision="mixed") as sim:
        sim.time_rk(steps)
        got = sim.solution()
    assert np.all(np.isfinite(got))
    rms = np.sqrt((ref * ref).mean(axis=0))
    sig = rms >= NOISE_FLOOR * rms.max()
    l2 = np.sqrt(((got - ref) ** 2).sum(axis=0) / np.maximum((ref * ref).sum(axis=0), 1e-300))
    linf = np.abs(got - ref).max(axis=0) / np.maximum(np.abs(ref).max(axis=0), 1e-300)
    print(f"mixed vs FP64, 4096^2, {steps} steps: rel L2 {l2[sig].max():.2e}, rel Linf {linf[sig].max():.2e}")
    assert l2[sig].max() <= MIXED_TOL
