"""Regenerate the golden fixtures of tests/golden/ from the reference.

Each fixture directory holds a complete input deck (written by
piafs_b200.cases with fixed seeds) and ``ref_final.bin``, the final solution
the reference CPU binary (serial build, oracle/_ref/PIAFS, compiled from the
llnl/piafs sources by oracle/Makefile) writes for it; decks that write the
photochemical species keep every species file the reference writes, renamed
``ref_op_species_z<k>_<NNNNN>.bin``.  Run from the repository root after
``make -C oracle``:

    python tests/golden/make_golden.py
"""
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from piafs_b200 import cases, deck  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "PIAFS")
DT2D = 0.4 / 2048   # CFL 0.4 at 2048^2 (sound speed 1 in the quiescent gas)
Z = deck.BoundaryZone
BIG = 1e99
# free stream rho = 1, u = 0.2, v = 0, p = 1/1.4 in conserved variables
FREE_02 = [1.0, 0.2, 0.0, (1 / 1.4) / 0.4 + 0.5 * 0.2 * 0.2]

CASES = {
    # the 1D Euler workload itself (N=1024, WENO5, Roe, SSPRK3, 1000 steps)
    "euler1d_weno5_roe_n1024": (cases.euler1d_density_wave, dict(N=1024, n_iter=1000, dt=1e-4)),
    "euler1d_crweno5_rusanov_mapped_n200": (cases.euler1d_density_wave, dict(
        N=200, n_iter=200, dt=1e-3, scheme="crweno5", upwinding="rusanov", weno={"mapped": 1})),
    "euler1d_weno5_llf_yc_rk4_n128": (cases.euler1d_density_wave, dict(
        N=128, n_iter=100, dt=2e-3, upwinding="llf-char", time_scheme_type="44", weno={"yc": 1})),
    "euler1d_crweno5_rf_borges_n97": (cases.euler1d_density_wave, dict(
        N=97, n_iter=60, dt=2e-3, amp=0.3, scheme="crweno5", upwinding="rf-char", weno={"borges": 1})),
    # the 2D photochemical workload at small size (same dt as at 2048^2); 60
    # steps carry the solution past the heating pulse (peak at t = 6.9e-3) so
    # that every conserved variable holds signal well above round-off
    "ns2d_chem_crweno5_llf_64x48": (cases.ns2d_photochem_beam, dict(N=64, NY=48, n_iter=60, dt=DT2D)),
    "ns2d_chem_weno5_llf_48x40": (cases.ns2d_photochem_beam, dict(N=48, NY=40, n_iter=60, dt=DT2D, scheme="weno5")),
    "ns2d_chem_crweno5_rf_borges_32x32": (cases.ns2d_photochem_beam, dict(
        N=32, NY=32, n_iter=60, dt=DT2D, upwinding="rf-char", weno={"borges": 1})),
    "ns2d_chem3layer_crweno5_llf_24x20": (cases.ns2d_photochem_beam, dict(
        N=24, NY=20, n_iter=60, dt=DT2D, extra_chem={"z_mm": 3.0, "nz": 20}, layers=3)),
    # species output (write_output yes): three layers, outputs at steps 0, 20, 40
    "ns2d_chem3layer_species_16x12": (cases.ns2d_photochem_beam, dict(
        N=16, NY=12, n_iter=40, dt=DT2D, extra_chem={"z_mm": 3.0, "nz": 20}, layers=3, write_output="yes",
        file_op_iter=20)),
    # WENO5 on characteristic variables (the reference's default interpolation)
    "euler1d_weno5char_roe_n256": (cases.euler1d_density_wave, dict(
        N=256, n_iter=200, dt=4e-4, interp="characteristic")),
    "euler1d_weno5char_llf_yc_n128": (cases.euler1d_density_wave, dict(
        N=128, n_iter=100, dt=2e-3, upwinding="llf-char", weno={"yc": 1}, interp="characteristic")),
    "ns2d_shear_weno5char_llf_re200_40x32": (cases.ns2d_shear_layer, dict(
        N=40, NY=32, n_iter=30, dt=2e-3, scheme="weno5", interp="characteristic")),
    "ns2d_chem_weno5char_rf_32x24": (cases.ns2d_photochem_beam, dict(
        N=32, NY=24, n_iter=60, dt=DT2D, scheme="weno5", upwinding="rf-char", interp="characteristic")),
    # CRWENO5 on characteristic variables (block-tridiagonal line solves;
    # models without photochemistry, where the reference's blocks invert)
    "euler1d_crweno5char_roe_n128": (cases.euler1d_density_wave, dict(
        N=128, n_iter=100, dt=2e-3, scheme="crweno5", interp="characteristic")),
    "euler1d_crweno5char_llf_mapped_n97": (cases.euler1d_density_wave, dict(
        N=97, n_iter=60, dt=2e-3, amp=0.3, scheme="crweno5", upwinding="llf-char", weno={"mapped": 1},
        interp="characteristic")),
    "ns2d_shear_crweno5char_llf_re200_40x32": (cases.ns2d_shear_layer, dict(
        N=40, NY=32, n_iter=30, dt=2e-3, interp="characteristic")),
    "ns2d_shear_crweno5char_rf_borges_36x28": (cases.ns2d_shear_layer, dict(
        N=36, NY=28, n_iter=30, dt=2e-3, upwinding="rf-char", weno={"borges": 1}, interp="characteristic")),
    # CRWENO5 lines longer than one CTA serves (thread-block clusters of 2-5
    # CTAs per line), 1D and 2D (long x lines; long y lines, the transposed pass)
    "euler1d_crweno5_roe_n6000": (cases.euler1d_density_wave, dict(N=6000, n_iter=100, dt=2e-5, scheme="crweno5")),
    "euler1d_crweno5_llf_yc_n20000": (cases.euler1d_density_wave, dict(
        N=20000, n_iter=60, dt=5e-6, scheme="crweno5", upwinding="llf-char", weno={"yc": 1})),
    "ns2d_shear_crweno5_llf_inviscid_4200x4": (cases.ns2d_shear_layer, dict(
        N=4200, NY=4, n_iter=20, dt=4e-5, Re=-1.0)),
    "ns2d_shear_crweno5_rf_inviscid_4x4500": (cases.ns2d_shear_layer, dict(
        N=4, NY=4500, n_iter=20, dt=4e-5, Re=-1.0, upwinding="rf-char")),
    # sponge zones (BCSponge.c): relaxation towards a reference state in a box
    "euler1d_weno5_roe_sponge_n200": (cases.euler1d_density_wave, dict(
        N=200, n_iter=100, dt=1e-3, sponge=dict(dim=0, face=1, extent=[0.7, 1.0], values=[1.0, 1.0, 3.0]))),
    "ns2d_shear_weno5_llf_sponge_40x32": (cases.ns2d_shear_layer, dict(
        N=40, NY=32, n_iter=30, dt=2e-3, scheme="weno5",
        sponge=dict(dim=1, face=-1, extent=[-1e9, 1e9, 0.0, 0.25], values=[1.0, 0.0, 0.0, 2.5]))),
    # the reference's remaining boundary conditions, fourth-order viscous
    # derivatives and the fifth-order upwind scheme, as its wall, inflow and
    # outflow examples use them (LidDrivenCavity, FlatPlateLaminar,
    # Uniform_Subsonic_Jet, Uniform_Supersonic_Jet)
    "ns2d_cavity_noslip_upw5_par4_32x32": (cases.ns2d_channel, dict(
        zones=[Z("noslip-wall", 0, 1, [0, 0, -BIG, BIG], [0.0, 0.0]),
               Z("noslip-wall", 0, -1, [0, 0, -BIG, BIG], [0.0, 0.0]),
               Z("noslip-wall", 1, 1, [-BIG, BIG, 0, 0], [0.0, 0.0]),
               Z("noslip-wall", 1, -1, [-BIG, BIG, 0, 0], [0.1, 0.0])],
        N=32, n_iter=100, dt=5e-3, scheme="upw5", Re=100.0, flow=(0.0, 0.0), bump=0.02)),
    "ns2d_flatplate_subsonic_weno5_par4_48x24": (cases.ns2d_channel, dict(
        zones=[Z("slip-wall", 1, 1, [0.0, 0.25, 0, 0], [0.0, 0.0]),
               Z("noslip-wall", 1, 1, [0.25, BIG, 0, 0], [0.0, 0.0]),
               Z("subsonic-outflow", 1, -1, [-BIG, BIG, 0, 0], values=[1 / 1.4]),
               Z("subsonic-inflow", 0, 1, [0, 0, -BIG, BIG], values=[1.0, 0.3, 0.0]),
               Z("subsonic-outflow", 0, -1, [0, 0, -BIG, BIG], values=[1 / 1.4])],
        N=48, NY=24, L=(1.0, 0.5), n_iter=60, dt=2e-3, bump_at=(0.5, 0.25))),
    "ns2d_ambivalent_dirichlet_weno5_llf_40x32": (cases.ns2d_channel, dict(
        zones=[Z("subsonic-ambivalent", 0, 1, [0, 0, -BIG, BIG], values=[1.0, 0.2, 0.0, 1 / 1.4]),
               Z("subsonic-ambivalent", 0, -1, [0, 0, -BIG, BIG], values=[1.0, 0.2, 0.0, 1 / 1.4]),
               Z("dirichlet", 1, 1, [-BIG, BIG, 0, 0], values=FREE_02),
               Z("dirichlet", 1, -1, [-BIG, BIG, 0, 0], values=FREE_02)],
        N=40, NY=32, n_iter=60, dt=2e-3, upwinding="llf-char", Re=500.0, par="2", time_scheme_type="ssprk3",
        flow=(0.2, 0.0))),
    "ns2d_chem_subsonic_jet_weno5char_rf_par4_24x32": (cases.ns2d_photochem_beam, dict(
        zones=[Z("periodic", 0, 1, [0, 0, -BIG, BIG]), Z("periodic", 0, -1, [0, 0, -BIG, BIG]),
               Z("subsonic-inflow", 1, 1, [-BIG, BIG, 0, 0], values=[1.0, 0.0, 0.05, 1.0, 0.01, 0, 0, 0, 0, 0]),
               Z("extrapolate", 1, -1, [-BIG, BIG, 0, 0])],
        N=24, NY=32, n_iter=60, dt=1e-3, scheme="weno5", upwinding="rf-char", interp="characteristic", par="4",
        flow=(0.0, 0.05))),
    "ns2d_chem_supersonic_jet_weno5_rf_24x32": (cases.ns2d_photochem_beam, dict(
        zones=[Z("periodic", 0, 1, [0, 0, -BIG, BIG]), Z("periodic", 0, -1, [0, 0, -BIG, BIG]),
               Z("supersonic-inflow", 1, 1, [-BIG, BIG, 0, 0],
                 values=[1.0, 0.0, 1.5, 1 / cases.chem_gamma(), 1.0, 0.005, 0, 0, 0, 0, 0]),
               Z("supersonic-outflow", 1, -1, [-BIG, BIG, 0, 0])],
        N=24, NY=32, n_iter=60, dt=1e-3, scheme="weno5", upwinding="rf-char", flow=(0.0, 1.5))),
    "euler1d_weno5_roe_dirichlet_n128": (cases.euler1d_density_wave, dict(
        zones=[Z("dirichlet", 0, 1, [0.0, 0.0], values=[1.0, 1.0, 1.0 / 0.4 + 0.5]),
               Z("extrapolate", 0, -1, [0.0, 0.0])],
        N=128, n_iter=100, dt=1e-3)),
    "ns2d_shear_crweno5_llf_re200_48x40": (cases.ns2d_shear_layer, dict(N=48, NY=40, n_iter=30, dt=2e-3)),
    "ns2d_shear_weno5_roe_re200_40x32": (cases.ns2d_shear_layer, dict(
        N=40, NY=32, n_iter=30, dt=2e-3, scheme="weno5", upwinding="roe")),
    "ns2d_shear_crweno5_rusanov_inviscid_32x36": (cases.ns2d_shear_layer, dict(
        N=32, NY=36, n_iter=30, dt=2e-3, upwinding="rusanov", Re=-1.0)),
}

KEEP = {"solver.inp", "boundary.inp", "physics.inp", "chemistry.inp", "weno.inp", "initial.inp", "imap.inp"}


def make(name):
    gen, kw = CASES[name]
    d = os.path.join(HERE, name)
    shutil.rmtree(d, ignore_errors=True)
    meta = gen(d, **kw)
    subprocess.run([REF], cwd=d, check=True, stdout=subprocess.DEVNULL)
    last = sorted(f for f in os.listdir(d) if re.fullmatch(r"op_\d+\.bin", f))[-1]
    os.replace(os.path.join(d, last), os.path.join(d, "ref_final.bin"))
    for f in os.listdir(d):
        if f.startswith("op_species_"):
            os.replace(os.path.join(d, f), os.path.join(d, "ref_" + f))
    for f in os.listdir(d):
        if f not in KEEP and f != "ref_final.bin" and not f.startswith("ref_op_species_"):
            os.remove(os.path.join(d, f))
    return meta


if __name__ == "__main__":
    if not os.path.exists(REF):
        sys.exit("build the reference first: make -C oracle")
    for n in (sys.argv[1:] or CASES):
        print(n, make(n))
