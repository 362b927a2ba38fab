"""The GPU path attached to the reference's own simulation objects
(include/piafs_hypar.h, libpiafs_hypar.so).

oracle/_ref/PIAFS_gpu is the reference binary -- its unmodified main,
initialisation, output and diagnostics, compiled from its own sources by
oracle/Makefile -- with TimeRK (TimeRK.c:34, the function
InitializeSolvers.c:204 stores in solver->TimeIntegrate) supplied by
oracle/dropin/timerk_gpu.c, which hands every step to piafs_gpu_TimeRK_ts.
The GPU state is mirrored from the reference's HyPar, physics, Chemistry and
boundary objects, never from the deck files.  Its output must match the
reference's own run of the deck (relative L2 per variable <= 1e-12, the
CompareSolutions-style norm of tests/test_gpu_parity.py).

oracle/_ref/PIAFS_gpu_check also holds each GPU operator, called through
the HyPar-signature entry points on the reference's host arrays, to the
reference's own operator on the state before the last step.
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from piafs_b200 import deck
from test_gpu_parity import assert_close

pytestmark = pytest.mark.gpu
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def binary(name):
    p = os.path.join(REF_DIR, name)
    if not os.access(p, os.X_OK):
        pytest.skip(f"{name} not built (make -C oracle dropin)")
    return p


def run(exe, d):
    r = subprocess.run([exe], cwd=d, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def copy_deck(name, dst):
    shutil.copytree(os.path.join(GOLDEN, name), dst,
                    ignore=shutil.ignore_patterns("ref_final.bin", "ref_op_species_*"))
    return dst


def final_op(d):
    return sorted(f for f in os.listdir(d) if re.fullmatch(r"op_\d{5}\.bin", f))[-1]


@pytest.mark.parametrize("name", ["ns2d_chem_crweno5_llf_64x48", "ns2d_shear_weno5_roe_re200_40x32",
                                  "euler1d_weno5_roe_n1024", "ns2d_chem_subsonic_jet_weno5char_rf_par4_24x32"])
def test_reference_binary_with_the_gpu_time_integrator(tmp_path, name):
    d = copy_deck(name, str(tmp_path / name))
    run(binary("PIAFS_gpu"), d)
    got = deck.read_op(os.path.join(d, final_op(d))).u
    assert_close(got, deck.read_op(os.path.join(GOLDEN, name, "ref_final.bin")).u, what=name)


def test_species_output_through_the_reference_binary(tmp_path):
    """With species output the photon density of the last RK stage comes
    back into the reference's Chemistry::nv_hnu before it writes the files."""
    name = "ns2d_chem3layer_species_16x12"
    d = copy_deck(name, str(tmp_path / name))
    run(binary("PIAFS_gpu"), d)
    src = os.path.join(GOLDEN, name)
    refs = sorted(f[len("ref_"):] for f in os.listdir(src) if f.startswith("ref_op_species_"))
    assert refs and sorted(f for f in os.listdir(d) if f.startswith("op_species_")) == refs
    for f in refs:
        ref = deck.read_op(os.path.join(src, "ref_" + f)).u
        got = deck.read_op(os.path.join(d, f)).u
        num = np.sqrt(((got - ref) ** 2).sum(axis=0))
        den = np.sqrt((ref ** 2).sum(axis=0))
        rel = np.where(den > 1e-15, num / np.maximum(den, 1e-300), num)
        assert rel.max() <= 1e-12, (f, rel)
    assert_close(deck.read_op(os.path.join(d, final_op(d))).u, deck.read_op(os.path.join(src, "ref_final.bin")).u)


def printed_diagnostics(out):
    """(iteration, CFL, norm) strings of the reference's TimePrintStep lines."""
    return re.findall(r"iter=\s*(\d+)\s+t=\S+\s+CFL=(\S+)\s+norm=(\S+)", out)


def test_diagnostics_and_counts_match_the_cpu_reference(tmp_path):
    """The reference computes CFL, residual norm and its call counts itself;
    through the GPU integrator the host state it computes them from is the
    GPU's, refreshed after every step it prints, and the printed lines and
    function_counts.dat equal those of the CPU run."""
    name = "ns2d_chem_crweno5_llf_64x48"
    dg = copy_deck(name, str(tmp_path / "gpu"))
    dc = copy_deck(name, str(tmp_path / "cpu"))
    for d in (dg, dc):
        txt = open(os.path.join(d, "solver.inp")).read()
        txt = re.sub(r"screen_op_iter\s+\d+", "screen_op_iter 5", txt)
        open(os.path.join(d, "solver.inp"), "w").write(txt)
    pg = printed_diagnostics(run(binary("PIAFS_gpu"), dg))
    pc = printed_diagnostics(run(binary("PIAFS"), dc))
    assert len(pg) == len(pc) == 12
    assert pg == pc
    assert open(os.path.join(dg, "function_counts.dat")).read() == open(os.path.join(dc, "function_counts.dat")).read()


OPERATOR_TOL = {
    # single evaluations of difference operators amplify interface rounding
    # by dxinv |f| / |df| (tests/test_gpu_parity.py); the pointwise ones do not
    "ApplyBoundaryConditions": 1e-15, "FFunction_0": 1e-14, "FFunction_1": 1e-14, "SourceFunction": 1e-12,
    "HyperbolicFunction": 1e-10, "ParabolicFunction": 1e-10, "RHSFunction": 1e-10,
}


@pytest.mark.parametrize("name", ["ns2d_chem_crweno5_llf_64x48", "ns2d_shear_crweno5_llf_re200_48x40",
                                  "ns2d_flatplate_subsonic_weno5_par4_48x24", "euler1d_crweno5_rusanov_mapped_n200"])
def test_hypar_signature_operators_match_the_reference(tmp_path, name):
    d = copy_deck(name, str(tmp_path / name))
    out = run(binary("PIAFS_gpu_check"), d)
    checks = dict((k, float(v)) for k, v in re.findall(r"^check (\S+) (\S+)$", out, re.M))
    assert {"ApplyBoundaryConditions", "HyperbolicFunction", "SourceFunction", "RHSFunction", "FFunction_0"} <= set(checks)
    for k, v in checks.items():
        assert v <= OPERATOR_TOL[k], (name, k, v)
