"""Synthetic input decks for the benchmark workloads.

Each generator writes a complete PIAFS input deck (solver.inp, boundary.inp,
physics.inp, optional chemistry.inp / weno.inp, binary initial.inp and
imap.inp) into a directory, in the reference's formats, so that the same
directory runs unchanged through the reference CPU binary and through this
package.  All inputs are synthetic and seeded (numpy ``default_rng``):
seed 0 drives field noise and beam amplitude, seed 1 ensemble parameters,
seed 2 serving arrivals, seed 3 serving request parameters.

Workloads:

* ``euler1d_density_wave`` -- 1D Euler, gamma 1.4, periodic [0,1) with
  x_i = i/N, rho = 1 + a sin(2 pi x), u = 1, p = 1; WENO5 (components), Roe,
  SSPRK3 with a fixed dt.
* ``ns2d_photochem_beam`` -- 2D Navier-Stokes with the O2/O3 photochemical
  heating source, periodic in x and slip walls in y, on [0,1]^2 with
  x_i = (i+1/2)/N; quiescent gas rho = 1 + U(-1e-6, 1e-6), u = v = 0,
  p = 1/gamma_chem; species O2 = 1, O3 = f_O3/f_O2, others 0; a Gaussian beam
  map A exp(-((x-1/2)^2+(y-1/2)^2)/r^2).  With chemistry on, the reference
  derives gamma, Re and Pr from chemistry.inp (NavierStokes2DInitialize.c:196-215);
  Re ~ 1e4 is realised through the beam half-angle theta (Re is proportional
  to 1/sin(theta): theta = 4.2117e-5 rad gives Re = 1.0e4).  dt is fixed from
  CFL 0.4 at t = 0 because the reference takes a fixed dt.
"""
from __future__ import annotations

import math
import os
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import deck

# Default chemistry gas properties (ChemistryInitialize.c: defaults), used to
# compute gamma_chem for the initial pressure and the CFL-based dt.
_CP_O2, _CV_O2 = 918.45, 650.0
THETA_RE_1E4 = 4.2117e-5


def _sponge_zones(sponge: Optional[Dict]):
    """The sponge zone of a deck, if any: dict(dim, face, extent, values)
    with extent = xmin, xmax per dimension and the reference state values
    (BCSponge.c: the solution is relaxed towards them inside the box)."""
    if not sponge:
        return []
    return [deck.BoundaryZone("sponge", sponge["dim"], sponge["face"], list(sponge["extent"]),
                              values=list(sponge["values"]))]


def chem_gamma(f_CO2: float = 0.0) -> float:
    """Specific-heat ratio of the O2/CO2 mixture (ChemistryInitialize.c:263-266)."""
    f_O2 = 1.0 - f_CO2
    cp = f_O2 * _CP_O2 + f_CO2 * 842.86
    cv = f_O2 * _CV_O2 + f_CO2 * 654.5
    return cp / cv


def euler1d_density_wave(path: str, N: int = 1024, n_iter: int = 1000, dt: float = 1e-4,
                         amp: float = 0.2, scheme: str = "weno5", upwinding: str = "roe",
                         time_scheme_type: str = "ssprk3", file_op_iter: Optional[int] = None,
                         op_file_format: str = "binary", weno: Optional[Dict] = None, interp: str = "components",
                         sponge: Optional[Dict] = None, zones: Optional[List[deck.BoundaryZone]] = None,
                         screen_op_iter: int = 0) -> Dict:
    """``zones`` replaces the periodic boundary zones."""
    os.makedirs(path, exist_ok=True)
    gamma = 1.4
    x = np.arange(N, dtype=np.float64) / N
    rho = 1.0 + amp * np.sin(2.0 * np.pi * x)
    uvel, p = 1.0, 1.0
    e = p / (gamma - 1.0) + 0.5 * rho * uvel * uvel
    u = np.stack([rho, rho * uvel, e], axis=1)
    deck.write_keyfile(os.path.join(path, "solver.inp"), {
        "ndims": 1, "nvars": 3, "size": N, "ghost": 3, "n_iter": n_iter,
        "time_scheme": "rk", "time_scheme_type": time_scheme_type,
        "hyp_space_scheme": scheme, "hyp_interp_type": interp, "dt": dt,
        "screen_op_iter": screen_op_iter or n_iter, "file_op_iter": file_op_iter or n_iter,
        "op_file_format": op_file_format, "ip_file_type": "binary", "op_overwrite": "no",
        "model": "euler1d",
    })
    deck.write_boundary(os.path.join(path, "boundary.inp"), (zones if zones is not None else [
        deck.BoundaryZone("periodic", 0, 1, [0.0, 0.0]),
        deck.BoundaryZone("periodic", 0, -1, [0.0, 0.0]),
    ]) + _sponge_zones(sponge))
    deck.write_keyfile(os.path.join(path, "physics.inp"), {"gamma": gamma, "upwinding": upwinding})
    if weno:
        deck.write_keyfile(os.path.join(path, "weno.inp"), weno)
    deck.write_array_binary(os.path.join(path, "initial.inp"), [x], u)
    return {"ndims": 1, "nvars": 3, "size": [N], "n_iter": n_iter, "dt": dt}


def ns2d_photochem_beam(path: str, N: int = 2048, NY: Optional[int] = None, n_iter: int = 200,
                        scheme: str = "crweno5", upwinding: str = "llf-char",
                        time_scheme_type: str = "ssprk3", seed: int = 0, beam_amp: Optional[float] = None,
                        beam_radius: float = 0.05, theta: float = THETA_RE_1E4, Re: float = 1e4,
                        cfl: float = 0.4, dt: Optional[float] = None, file_op_iter: Optional[int] = None,
                        op_file_format: str = "binary", chemistry: bool = True,
                        noise: float = 1e-6, weno: Optional[Dict] = None, extra_chem: Optional[Dict] = None,
                        interp: str = "components",
                        screen_op_iter: int = 0, write_output: str = "no", layers: int = 1,
                        zones: Optional[List[deck.BoundaryZone]] = None, par: str = "2",
                        flow: Sequence[float] = (0.0, 0.0)) -> Dict:
    """``layers`` is the number of simulated z-layers, z_i + 1 with
    z_i = ceil(z_mm 1e-3 nz / Lz) from chemistry.inp (ChemistryInitialize.c:353);
    each layer carries its own 7 species.  ``zones`` replaces the boundary
    zones (periodic in x, slip walls in y), ``par`` is par_space_scheme and
    ``flow`` the initial velocity (u, v)."""
    os.makedirs(path, exist_ok=True)
    NX = N
    NY = NY or N
    rng = np.random.default_rng(seed)
    gamma = chem_gamma() if chemistry else 1.4
    nvars = 4 + 7 * layers if chemistry else 4
    x = (np.arange(NX, dtype=np.float64) + 0.5) / NX
    y = (np.arange(NY, dtype=np.float64) + 0.5) / NY
    rho = 1.0 + rng.uniform(-noise, noise, size=(NY, NX))
    p = 1.0 / gamma
    u = np.zeros((NY, NX, nvars))
    u0, v0 = float(flow[0]), float(flow[1])
    u[..., 0] = rho
    u[..., 1] = rho * u0
    u[..., 2] = rho * v0
    u[..., 3] = p / (gamma - 1.0) + 0.5 * rho * (u0 * u0 + v0 * v0)
    if chemistry:
        for iz in range(layers):
            u[..., 4 + 7 * iz] = 1.0            # O2 (normalised by n_O2)
            u[..., 5 + 7 * iz] = 0.005 / 1.0    # O3 = f_O3 / f_O2
    A = float(rng.uniform(0.5, 1.5)) if beam_amp is None else float(beam_amp)
    X, Y = np.meshgrid(x, y)
    imap = A * np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / beam_radius ** 2)
    c0 = math.sqrt(gamma * p / (1.0 + noise))
    if dt is None:
        dt = cfl * (1.0 / max(NX, NY)) / c0
    deck.write_keyfile(os.path.join(path, "solver.inp"), {
        "ndims": 2, "nvars": nvars, "size": [NX, NY], "ghost": 3, "n_iter": n_iter,
        "time_scheme": "rk", "time_scheme_type": time_scheme_type,
        "hyp_space_scheme": scheme, "hyp_interp_type": interp,
        "par_space_scheme": par, "dt": dt,
        "screen_op_iter": screen_op_iter or n_iter, "file_op_iter": file_op_iter or n_iter,
        "op_file_format": op_file_format, "ip_file_type": "binary", "op_overwrite": "no",
        "model": "navierstokes2d",
    })
    big = 1e99
    deck.write_boundary(os.path.join(path, "boundary.inp"), zones if zones is not None else [
        deck.BoundaryZone("periodic", 0, 1, [0.0, 0.0, -big, big]),
        deck.BoundaryZone("periodic", 0, -1, [0.0, 0.0, -big, big]),
        deck.BoundaryZone("slip-wall", 1, 1, [-big, big, 0.0, 0.0], [0.0, 0.0]),
        deck.BoundaryZone("slip-wall", 1, -1, [-big, big, 0.0, 0.0], [0.0, 0.0]),
    ])
    phys = {"gamma": 1.4, "upwinding": upwinding, "Pr": 0.72, "Re": Re,
            "include_chemistry": "yes" if chemistry else "no", "write_output": write_output}
    deck.write_keyfile(os.path.join(path, "physics.inp"), phys)
    if chemistry:
        chem = {"theta": theta}
        if extra_chem:
            chem.update(extra_chem)
        deck.write_keyfile(os.path.join(path, "chemistry.inp"), chem)
        deck.write_array_binary(os.path.join(path, "imap.inp"), [x, y], imap.reshape(-1, 1))
    if weno:
        deck.write_keyfile(os.path.join(path, "weno.inp"), weno)
    deck.write_array_binary(os.path.join(path, "initial.inp"), [x, y], u.reshape(-1, nvars))
    return {"ndims": 2, "nvars": nvars, "size": [NX, NY], "n_iter": n_iter, "dt": dt,
            "beam_amp": A, "gamma": gamma}


def ns2d_shear_layer(path: str, N: int = 64, NY: Optional[int] = None, n_iter: int = 20, dt: float = 2e-3,
                     scheme: str = "crweno5", upwinding: str = "llf-char", Re: float = 200.0,
                     time_scheme_type: str = "ssprk3", weno: Optional[Dict] = None, delta: float = 0.05,
                     amp: float = 0.05, file_op_iter: Optional[int] = None, op_file_format: str = "binary",
                     screen_op_iter: int = 0, interp: str = "components", sponge: Optional[Dict] = None) -> Dict:
    """2D Navier-Stokes (no chemistry) double shear layer, periodic in x, slip
    walls in y: u = tanh((y-1/4)/delta) - tanh((y-3/4)/delta) - 1,
    v = amp sin(2 pi x), rho = 1, p = 1/gamma; Re from physics.inp."""
    os.makedirs(path, exist_ok=True)
    NX, NY = N, NY or N
    gamma = 1.4
    x = (np.arange(NX, dtype=np.float64) + 0.5) / NX
    y = (np.arange(NY, dtype=np.float64) + 0.5) / NY
    X, Y = np.meshgrid(x, y)
    uu = np.tanh((Y - 0.25) / delta) - np.tanh((Y - 0.75) / delta) - 1.0
    vv = amp * np.sin(2 * np.pi * X)
    rho = np.ones_like(X)
    p = 1.0 / gamma
    u = np.zeros((NY, NX, 4))
    u[..., 0] = rho
    u[..., 1] = rho * uu
    u[..., 2] = rho * vv
    u[..., 3] = p / (gamma - 1.0) + 0.5 * rho * (uu * uu + vv * vv)
    deck.write_keyfile(os.path.join(path, "solver.inp"), {
        "ndims": 2, "nvars": 4, "size": [NX, NY], "ghost": 3, "n_iter": n_iter,
        "time_scheme": "rk", "time_scheme_type": time_scheme_type,
        "hyp_space_scheme": scheme, "hyp_interp_type": interp, "par_space_scheme": "2",
        "dt": dt, "screen_op_iter": screen_op_iter or n_iter, "file_op_iter": file_op_iter or n_iter,
        "op_file_format": op_file_format, "ip_file_type": "binary", "op_overwrite": "no",
        "model": "navierstokes2d",
    })
    big = 1e99
    deck.write_boundary(os.path.join(path, "boundary.inp"), [
        deck.BoundaryZone("periodic", 0, 1, [0.0, 0.0, -big, big]),
        deck.BoundaryZone("periodic", 0, -1, [0.0, 0.0, -big, big]),
        deck.BoundaryZone("slip-wall", 1, 1, [-big, big, 0.0, 0.0], [0.0, 0.0]),
        deck.BoundaryZone("slip-wall", 1, -1, [-big, big, 0.0, 0.0], [0.0, 0.0]),
    ] + _sponge_zones(sponge) + [
    ])
    deck.write_keyfile(os.path.join(path, "physics.inp"), {"gamma": gamma, "upwinding": upwinding, "Re": Re,
                                                           "Pr": 0.72})
    if weno:
        deck.write_keyfile(os.path.join(path, "weno.inp"), weno)
    deck.write_array_binary(os.path.join(path, "initial.inp"), [x, y], u.reshape(-1, 4))
    return {"ndims": 2, "nvars": 4, "size": [NX, NY], "n_iter": n_iter, "dt": dt}


def ns2d_density_wave(path: str, N: int = 64, NY: Optional[int] = None, axis: int = 0, n_iter: int = 10,
                      dt: float = 1e-4, amp: float = 0.2, scheme: str = "crweno5", upwinding: str = "llf-char",
                      Re: float = 100.0, time_scheme_type: str = "ssprk3", op_file_format: str = "binary",
                      file_op_iter: Optional[int] = None, screen_op_iter: int = 0) -> Dict:
    """2D Navier-Stokes (no chemistry) density wave along `axis`, periodic in
    both directions: rho = 1 + amp sin(2 pi s), velocity 1 along the wave,
    p = 1/gamma, where s is x (axis 0) or y (axis 1)."""
    os.makedirs(path, exist_ok=True)
    NX, NY = N, NY or N
    gamma = 1.4
    x = np.arange(NX, dtype=np.float64) / NX
    y = np.arange(NY, dtype=np.float64) / NY
    X, Y = np.meshgrid(x, y)
    S = X if axis == 0 else Y
    rho = 1.0 + amp * np.sin(2 * np.pi * S)
    p = 1.0 / gamma
    u = np.zeros((NY, NX, 4))
    u[..., 0] = rho
    u[..., 1 + axis] = rho
    u[..., 3] = p / (gamma - 1.0) + 0.5 * rho
    deck.write_keyfile(os.path.join(path, "solver.inp"), {
        "ndims": 2, "nvars": 4, "size": [NX, NY], "ghost": 3, "n_iter": n_iter,
        "time_scheme": "rk", "time_scheme_type": time_scheme_type,
        "hyp_space_scheme": scheme, "hyp_interp_type": "components", "par_space_scheme": "2",
        "dt": dt, "screen_op_iter": screen_op_iter or n_iter, "file_op_iter": file_op_iter or n_iter,
        "op_file_format": op_file_format, "ip_file_type": "binary", "op_overwrite": "no",
        "model": "navierstokes2d",
    })
    deck.write_boundary(os.path.join(path, "boundary.inp"), [
        deck.BoundaryZone("periodic", 0, 1, [0.0, 0.0, -1e99, 1e99]),
        deck.BoundaryZone("periodic", 0, -1, [0.0, 0.0, -1e99, 1e99]),
        deck.BoundaryZone("periodic", 1, 1, [-1e99, 1e99, 0.0, 0.0]),
        deck.BoundaryZone("periodic", 1, -1, [-1e99, 1e99, 0.0, 0.0]),
    ])
    deck.write_keyfile(os.path.join(path, "physics.inp"), {"gamma": gamma, "upwinding": upwinding, "Re": Re,
                                                           "Pr": 0.72})
    deck.write_array_binary(os.path.join(path, "initial.inp"), [x, y], u.reshape(-1, 4))
    return {"ndims": 2, "nvars": 4, "size": [NX, NY], "n_iter": n_iter, "dt": dt}


def ns2d_channel(path: str, zones: List[deck.BoundaryZone], N: int = 48, NY: Optional[int] = None,
                 L: Sequence[float] = (1.0, 1.0), n_iter: int = 50, dt: float = 2e-3, scheme: str = "weno5",
                 upwinding: str = "roe", interp: str = "components", Re: float = 1000.0, Pr: float = 0.72,
                 par: str = "4", time_scheme_type: str = "44", flow: Sequence[float] = (0.3, 0.0),
                 rho0: float = 1.0, bump: float = 0.05, bump_at: Sequence[float] = (0.5, 0.5),
                 bump_radius: float = 0.1, file_op_iter: Optional[int] = None, op_file_format: str = "binary",
                 screen_op_iter: int = 0) -> Dict:
    """2D Navier-Stokes (no chemistry) on [0, L0] x [0, L1] with x_i = (i+1/2) L0/N
    and the given boundary zones: a uniform flow (rho0, u, v, p = 1/gamma)
    with a Gaussian density bump of relative height ``bump`` at ``bump_at``
    (pressure uniform), as in the reference's wall, inflow and outflow
    examples (flat plate, lid-driven cavity)."""
    os.makedirs(path, exist_ok=True)
    NX, NY = N, NY or N
    gamma = 1.4
    x = (np.arange(NX, dtype=np.float64) + 0.5) * (L[0] / NX)
    y = (np.arange(NY, dtype=np.float64) + 0.5) * (L[1] / NY)
    X, Y = np.meshgrid(x, y)
    rho = rho0 * (1.0 + bump * np.exp(-((X - bump_at[0]) ** 2 + (Y - bump_at[1]) ** 2) / bump_radius ** 2))
    uu, vv = float(flow[0]), float(flow[1])
    p = 1.0 / gamma
    u = np.zeros((NY, NX, 4))
    u[..., 0] = rho
    u[..., 1] = rho * uu
    u[..., 2] = rho * vv
    u[..., 3] = p / (gamma - 1.0) + 0.5 * rho * (uu * uu + vv * vv)
    deck.write_keyfile(os.path.join(path, "solver.inp"), {
        "ndims": 2, "nvars": 4, "size": [NX, NY], "ghost": 3, "n_iter": n_iter,
        "time_scheme": "rk", "time_scheme_type": time_scheme_type,
        "hyp_space_scheme": scheme, "hyp_interp_type": interp, "par_space_scheme": par,
        "dt": dt, "screen_op_iter": screen_op_iter or n_iter, "file_op_iter": file_op_iter or n_iter,
        "op_file_format": op_file_format, "ip_file_type": "binary", "op_overwrite": "no",
        "model": "navierstokes2d",
    })
    deck.write_boundary(os.path.join(path, "boundary.inp"), zones)
    deck.write_keyfile(os.path.join(path, "physics.inp"), {"gamma": gamma, "upwinding": upwinding, "Re": Re,
                                                           "Pr": Pr})
    deck.write_array_binary(os.path.join(path, "initial.inp"), [x, y], u.reshape(-1, 4))
    return {"ndims": 2, "nvars": 4, "size": [NX, NY], "n_iter": n_iter, "dt": dt}


def ensemble_params(n: int = 256, steps: int = 100, seed: int = 1, side_range=(64, 512),
                    dt: float = 0.4 / 2048):
    """The member parameters of ``ensemble`` (no files written): per member
    its index, grid side, beam amplitude and radius, Re, beam half-angle and
    time step, drawn in member order from ``seed``."""
    rng = np.random.default_rng(seed)
    lo, hi = side_range
    out = []
    for k in range(n):
        side = int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))) / 32.0)) * 32
        side = min(max(side, 32 * math.ceil(lo / 32)), hi)
        amp = float(rng.uniform(0.5, 1.5))
        radius = float(rng.uniform(0.02, 0.1))
        Re = float(math.exp(rng.uniform(math.log(1e3), math.log(1e5))))
        theta = math.asin(min(1.0, math.sin(THETA_RE_1E4) * 1e4 / Re))
        mdt = min(0.4 / side, dt * 1e4 / Re, 0.1 * Re / (side * side))
        out.append({"index": k, "side": side, "beam_amp": amp, "beam_radius": radius, "Re": Re, "theta": theta,
                    "steps": steps, "dt": mdt})
    return out


def ensemble(root: str, n: int = 256, steps: int = 100, seed: int = 1, side_range=(64, 512),
             dt: float = 0.4 / 2048, op_file_format: str = "none", members=None):
    """The batched-ensemble workload: ``n`` independent 2D photochemical
    Navier-Stokes members (``ns2d_photochem_beam`` decks) with grid sides
    drawn log-uniformly in ``side_range`` and rounded to multiples of 32, beam
    amplitude U(0.5, 1.5), beam 1/e radius U(0.02, 0.1) and Re log-uniform in
    [1e3, 1e5] (realised through the beam half-angle, Re ~ 1/sin(theta));
    WENO5, LLF, SSPRK3, ``steps`` steps.  The normalised heating pulse
    shortens as 1/Re (the half-angle sets the acoustic time scale), and
    explicit viscosity bounds dt by the diffusion number, so each member takes
    dt = min(0.4 dx, dt_2048 * 1e4 / Re, 0.1 Re dx^2) with dx = 1/side: CFL
    0.4, capped at the pulse resolution of the 2048^2 workload at Re = 1e4
    (dt_2048 = 0.4/2048, about 35 steps per pulse width) and at a diffusion
    number nu dt / dx^2 of about 0.2 for the thermal diffusivity
    gamma / (Pr Re).  Member k's field noise uses seed 1000 * seed + k.
    ``members`` (indices) restricts the decks written and returned to a
    subset; member k is the same whichever subset it is written in.  Returns
    the ``ensemble_params`` dicts of the written members with their "dir"."""
    keep = None if members is None else set(int(k) for k in members)
    out = []
    for m in ensemble_params(n, steps, seed, side_range, dt):
        k = m["index"]
        if keep is not None and k not in keep:
            continue
        d = os.path.join(root, f"member{k:04d}")
        ns2d_photochem_beam(d, N=m["side"], n_iter=steps, scheme="weno5", seed=1000 * seed + k,
                            beam_amp=m["beam_amp"], beam_radius=m["beam_radius"], theta=m["theta"], Re=m["Re"],
                            dt=m["dt"], op_file_format=op_file_format)
        out.append(dict(m, dir=d))
    return out


def serving_trace(n: int = 10000, rate: float = 2000.0, frac_1d: float = 0.7, seed_arrivals: int = 2,
                  seed_params: int = 3, n1d=(256, 8192), side2d=(64, 1024), steps=(50, 500)):
    """The request-serving workload: ``n`` requests arriving as a Poisson
    process of ``rate`` requests/s (seed 2).  A fraction ``frac_1d`` are 1D
    Euler density waves (N log-uniform in ``n1d``, amplitude U(0.05, 0.3),
    dt = 0.1/N as in the 1024-point case), the rest 2D photochemical beams
    (side log-uniform in ``side2d``, beam parameters and dt as in
    ``ensemble``, density noise 1e-6); each runs a uniform number of SSPRK3
    steps in ``steps`` (parameters: seed 3).  Returns (requests, arrivals):
    dicts with the fields of piafs_gpu_request, and arrival times in seconds."""
    ra = np.random.default_rng(seed_arrivals)
    arrivals = np.cumsum(ra.exponential(1.0 / rate, size=n))
    rp = np.random.default_rng(seed_params)
    reqs = []
    for k in range(n):
        nsteps = int(rp.integers(steps[0], steps[1] + 1))
        if rp.uniform() < frac_1d:
            N = int(round(math.exp(rp.uniform(math.log(n1d[0]), math.log(n1d[1])))))
            reqs.append({"kind": 1, "n": N, "nsteps": nsteps, "dt": 0.1 / N, "amp": float(rp.uniform(0.05, 0.3)),
                         "beam_radius": 0.0, "Re": 0.0, "noise": 0.0, "seed": 0})
        else:
            side = int(round(math.exp(rp.uniform(math.log(side2d[0]), math.log(side2d[1])))))
            amp = float(rp.uniform(0.5, 1.5))
            radius = float(rp.uniform(0.02, 0.1))
            Re = float(math.exp(rp.uniform(math.log(1e3), math.log(1e5))))
            dt = min(0.4 / side, (0.4 / 2048) * 1e4 / Re, 0.1 * Re / (side * side))
            reqs.append({"kind": 2, "n": side, "nsteps": nsteps, "dt": dt, "amp": amp, "beam_radius": radius,
                         "Re": Re, "noise": 1e-6, "seed": 1000003 * seed_params + k})
    return reqs, arrivals
