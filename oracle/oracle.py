"""Python front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Reads a PIAFS input deck the way the reference does and sets up the arrays
and parameters the C restatement (piafs_oracle.c) needs:

* solver.inp defaults and keys           src/Simulation/ReadInputs.c:202-450
* physics.inp (NS2D / Euler1D)           NavierStokes2DInitialize.c:68-235,
                                         Euler1DInitialize.c:58-170
* chemistry.inp + normalisation          ChemistryInitialize.c:69-481
* weno.inp                               WENOInitialize.c:29-183
* grid ghosts by linear extrapolation    ReadArray.c:71-91
* dxinv = 2/(x[i+1]-x[i-1]), ghost copy  InitialSolution.c:73-113
* boundary zone extents (FindInterval)   InitializeBoundaries.c:296-378,
                                         FindInterval.c:21-50
* Butcher tableaux                       TimeExplicitRKInitialize.c:25-95

The oracle is a checker: only tests, the smoke check and the benchmark's CPU
baseline use it.  It is never the product path.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liborc_piafs.so")
MAXZ = 16


class OrcParams(C.Structure):
    _fields_ = [
        ("ndims", C.c_int), ("nvars", C.c_int), ("ghosts", C.c_int), ("dim", C.c_int * 2),
        ("model", C.c_int), ("scheme", C.c_int), ("upwind", C.c_int), ("weno_type", C.c_int),
        ("no_limiting", C.c_int), ("weno_eps", C.c_double),
        ("gamma", C.c_double), ("Re", C.c_double), ("Pr", C.c_double), ("Tref", C.c_double),
        ("T0", C.c_double), ("TS", C.c_double), ("TA", C.c_double), ("TB", C.c_double),
        ("bc_gamma", C.c_double), ("viscous", C.c_int),
        ("include_chem", C.c_int), ("n_flow_vars", C.c_int), ("nz", C.c_int), ("z_stride", C.c_int),
        ("grid_stride", C.c_int),
        ("k", C.c_double * 11), ("q", C.c_double * 11),
        ("chem_gamma", C.c_double), ("I0", C.c_double), ("c", C.c_double), ("h", C.c_double),
        ("nu", C.c_double), ("n_O2", C.c_double), ("t_start_norm", C.c_double),
        ("t_pulse_norm", C.c_double), ("sO3", C.c_double), ("dz", C.c_double),
        ("nstages", C.c_int), ("A", C.c_double * 16), ("b", C.c_double * 4), ("cst", C.c_double * 4),
        ("dt", C.c_double),
        ("nb", C.c_int), ("bc_type", C.c_int * MAXZ), ("bc_dim", C.c_int * MAXZ),
        ("bc_face", C.c_int * MAXZ), ("bc_is", (C.c_int * 2) * MAXZ), ("bc_ie", (C.c_int * 2) * MAXZ),
        ("bc_vel", (C.c_double * 2) * MAXZ),
    ]


def build(force: bool = False) -> str:
    """Compile the restatement into oracle/liborc_piafs.so (gcc -O2, no FMA)."""
    src = os.path.join(HERE, "piafs_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-std=c99", "-O2", "-fPIC", "-shared", "-o", LIB, src, "-lm"])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        dp = C.POINTER(C.c_double)
        pp = C.POINTER(OrcParams)
        L.orc_run.argtypes = [pp, dp, dp, dp, C.c_double, C.c_int]
        L.orc_rhs.argtypes = [pp, dp, dp, dp, dp, C.c_double]
        L.orc_hyperbolic.argtypes = [pp, dp, dp, dp]
        L.orc_parabolic.argtypes = [pp, dp, dp, dp]
        L.orc_source.argtypes = [pp, dp, dp, dp, C.c_double]
        L.orc_apply_bc.argtypes = [pp, dp]
        L.orc_flux.argtypes = [pp, dp, dp, C.c_int]
        L.orc_interp.argtypes = [pp, dp, dp, dp, C.c_int, C.c_int, C.c_int]
        L.orc_upwind.argtypes = [pp, dp, dp, dp, dp, dp, dp, C.c_int]
        L.orc_first_derivative.argtypes = [pp, dp, dp, C.c_int, C.c_int, C.c_int]
        L.orc_tridiag.argtypes = [dp, dp, dp, dp, C.c_int, C.c_int]
        L.orc_cfl.argtypes = [pp, dp, dp]
        L.orc_cfl.restype = C.c_double
        L.orc_ninterfaces.argtypes = [pp, C.c_int]
        L.orc_ninterfaces.restype = C.c_long
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


# ------------------------------------------------------------------ parsing
def _keyfile(path):
    if not os.path.exists(path):
        return None
    toks = open(path).read().split()
    if not toks or toks[0] != "begin":
        raise ValueError(f"{path}: illegal format")
    out, i = {}, 1
    while i < len(toks) and toks[i] != "end":
        k = toks[i]
        i += 1
        if k in ("size", "size_exact", "iproc"):
            vals = []
            while i < len(toks) and toks[i] != "end":
                try:
                    float(toks[i])
                except ValueError:
                    break
                vals.append(toks[i])
                i += 1
            out[k] = vals
        else:
            out[k] = toks[i]
            i += 1
    return out


def _find_interval(a, b, x):
    """FindInterval.c:21-50 (x = interior coordinates of one dimension)."""
    N = len(x)
    imax, imin = -1, N
    min_dx = x[1] - x[0] if N > 1 else 1.0
    for i in range(2, N):
        dx = x[i] - x[i - 1]
        if dx < min_dx:
            min_dx = dx
    tol = 1e-10 * min_dx
    for i in range(N):
        if x[i] <= b + tol:
            imax = i + 1
    for i in range(N - 1, -1, -1):
        if x[i] >= a - tol:
            imin = i
    return imin, imax


def _tableau(time_scheme, ttype):
    """TimeExplicitRKInitialize.c:25-95 (and forward Euler)."""
    if time_scheme == "euler":
        return 1, [0.0], [1.0], [0.0]
    if ttype == "1fe":
        return 1, [0.0], [1.0], [0.0]
    if ttype == "22":
        return 2, [0, 0, 1.0, 0], [0.5, 0.5], [0, 1.0]
    if ttype == "33":
        A = [0.0] * 9
        A[3] = 2.0 / 3.0; A[6] = 2.0 / 3.0 - 1.0 / 4.0; A[7] = 1.0 / 4.0
        return 3, A, [1.0 / 4.0, -1.0 / 4.0, 1.0], [0, 2.0 / 3.0, 2.0 / 3.0]
    if ttype == "44":
        A = [0.0] * 16
        A[4] = 0.5; A[9] = 0.5; A[14] = 1.0
        return 4, A, [1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0], [0, 0.5, 0.5, 1.0]
    if ttype in ("ssprk3", "tvdrk3"):
        A = [0.0] * 9
        A[3] = 1.0; A[6] = 0.25; A[7] = 0.25
        return 3, A, [1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0], [0, 1.0, 0.5]
    raise ValueError(f"unsupported RK type {ttype}")


class Case:
    """A deck loaded into oracle arrays (AoS, ghosts included)."""

    def __init__(self, path: str):
        self.path = path
        s = _keyfile(os.path.join(path, "solver.inp"))
        ndims = int(s.get("ndims", 1))
        nvars = int(s.get("nvars", 1))
        g = int(s.get("ghost", 1))
        dims = [int(v) for v in s["size"]]
        self.ndims, self.nvars, self.ghosts, self.dims = ndims, nvars, g, dims
        self.n_iter = int(s.get("n_iter", 0))
        self.dt = float(s.get("dt", 0.0))
        self.model = s.get("model", "none")
        scheme = s.get("hyp_space_scheme", "1")
        interp = s.get("hyp_interp_type", "characteristic")
        if interp != "components" and nvars > 1:
            raise ValueError("oracle restates the component-wise interpolation only")
        P = OrcParams()
        P.ndims, P.nvars, P.ghosts = ndims, nvars, g
        P.dim[0] = dims[0]
        P.dim[1] = dims[1] if ndims == 2 else 1
        P.scheme = {"weno5": 0, "crweno5": 1}[scheme]
        P.model = {"euler1d": 0, "navierstokes2d": 1}[self.model]
        # weno.inp (WENOInitialize.c:46-90)
        w = _keyfile(os.path.join(path, "weno.inp")) or {}
        P.no_limiting = int(w.get("no_limiting", 0))
        P.weno_eps = float(w.get("epsilon", 1e-6))
        if int(w.get("yc", 0)):
            P.weno_type = 3
        elif int(w.get("borges", 0)):
            P.weno_type = 2
        elif int(w.get("mapped", 0)):
            P.weno_type = 1
        else:
            P.weno_type = 0
        # physics.inp
        ph = _keyfile(os.path.join(path, "physics.inp")) or {}
        gamma = float(ph.get("gamma", 1.4))
        # wall BCs keep the physics.inp gamma (set before chemistry overrides
        # it, NavierStokes2DInitialize.c:172-174); Euler1D never sets it (0)
        P.bc_gamma = gamma if self.model == "navierstokes2d" else 0.0
        upw = ph.get("upwinding", "roe")
        P.upwind = {"roe": 0, "rf-char": 1, "llf-char": 2, "rusanov": 3}[upw]
        include_chem = ph.get("include_chemistry", "no") == "yes"
        Re = float(ph.get("Re", -1.0))
        Pr = float(ph.get("Pr", 0.72))
        Tref = float(ph.get("T_ref", 273.15))
        T0 = float(ph.get("T_0", 275.0))
        TS = float(ph.get("T_S", 110.4))
        TA = float(ph.get("T_A", 245.4))
        TB = float(ph.get("T_B", 27.6))
        nflow = 4 if P.model == 1 else 3
        P.include_chem = int(include_chem)
        P.n_flow_vars = nflow
        self.chem = None
        if include_chem:
            ch = self._chemistry(path, nflow)
            self.chem = ch
            gamma = ch["gamma"]
            if P.model == 1:
                Tref = ch["Ti"]
                if Re > 0:
                    # NavierStokes2DInitialize.c:203-215
                    mu_ref = ch["mu0"] * math.exp(1.5 * math.log(ch["Ti"] / T0)) * ((T0 + TS) / (ch["Ti"] + TS))
                    kappa_ref = (ch["kappa0"] * math.exp(1.5 * math.log(ch["Ti"] / T0))
                                 * ((T0 + TA * math.exp(-TB / T0)) / (ch["Ti"] + TA * math.exp(-TB / ch["Ti"]))))
                    Re = ch["rho_ref"] * ch["v_ref"] * ch["L_ref"] / mu_ref
                    Pr = ch["gamma"] * ch["R"] / (ch["gamma"] - 1) * mu_ref / kappa_ref
            P.nz = ch["nz"]
            P.z_stride = 7
            P.grid_stride = nvars
            for i, key in enumerate(["k0a", "k0b", "k1a", "k1b", "k2a", "k2b", "k3a", "k3b", "k4", "k5", "k6"]):
                P.k[i] = ch[key + "_norm"]
            for i, key in enumerate(["q0a", "q0b", "q1a", "q1b", "q2a", "q2b", "q3a", "q3b", "q4", "q5", "q6"]):
                P.q[i] = ch[key + "_norm"]
            P.chem_gamma = ch["gamma"]
            P.I0, P.c, P.h, P.nu, P.n_O2 = ch["I0"], ch["c"], ch["h"], ch["nu"], ch["n_O2"]
            P.t_start_norm, P.t_pulse_norm = ch["t_start_norm"], ch["t_pulse_norm"]
            P.sO3, P.dz = ch["sO3"], ch["dz"]
            if nvars != nflow + 7 * ch["nz"]:
                raise ValueError("nvars inconsistent with chemistry layers")
        P.gamma, P.Re, P.Pr, P.Tref, P.T0, P.TS, P.TA, P.TB = gamma, Re, Pr, Tref, T0, TS, TA, TB
        P.viscous = int(P.model == 1 and Re > 0)
        self.gamma, self.Re, self.Pr = gamma, Re, Pr
        ns, A, b, c = _tableau(s.get("time_scheme", "euler"), s.get("time_scheme_type", " "))
        P.nstages = ns
        for i, v in enumerate(A):
            P.A[i] = v
        for i, v in enumerate(b):
            P.b[i] = v
        for i, v in enumerate(c):
            P.cst[i] = v
        P.dt = self.dt
        # grid + initial solution (ReadArray.c)
        npts = int(np.prod(dims))
        raw = np.fromfile(os.path.join(path, "initial.inp"), dtype=np.float64)
        xs, off = [], 0
        for d in dims:
            xs.append(raw[off:off + d].copy())
            off += d
        uint = raw[off:off + npts * nvars].reshape(npts, nvars)
        self.grid = xs
        self.x = np.concatenate([self._ghost_x(xi) for xi in xs])
        self.dxinv = np.concatenate([self._dxinv(self._ghost_x(xi), len(xi)) for xi in xs])
        W0 = dims[0] + 2 * g
        W1 = dims[1] + 2 * g if ndims == 2 else 1
        self.shape_g = (W1, W0)
        u = np.zeros((W1, W0, nvars))
        if ndims == 2:
            u[g:g + dims[1], g:g + dims[0], :] = uint.reshape(dims[1], dims[0], nvars)
        else:
            u[0, g:g + dims[0], :] = uint
        self.u0 = np.ascontiguousarray(u.reshape(-1))
        # intensity map (ChemistryInitialize.c:441-476)
        imap = np.zeros((W1, W0))
        if include_chem:
            fn = os.path.join(path, "imap.inp")
            if os.path.exists(fn):
                rawm = np.fromfile(fn, dtype=np.float64)
                vals = rawm[sum(dims):sum(dims) + npts]
                if ndims == 2:
                    imap[g:g + dims[1], g:g + dims[0]] = vals.reshape(dims[1], dims[0])
                else:
                    imap[0, g:g + dims[0]] = vals
            else:
                ch = self.chem
                x0 = xs[0][0]
                xx = xs[0]
                val = ch["IA"] + ch["IB"] * np.cos(ch["kg"] * ch["L_ref"] * (xx - x0) * (1.0 - ch["IC"] * (xx - x0)))
                if ndims == 2:
                    imap[g:g + dims[1], g:g + dims[0]] = val[None, :]
                else:
                    imap[0, g:g + dims[0]] = val
        self.imap = np.ascontiguousarray(imap.reshape(-1))
        # boundary zones
        toks = open(os.path.join(path, "boundary.inp")).read().split()
        nb, i = int(toks[0]), 1
        P.nb = nb
        for n in range(nb):
            bt, dim, face = toks[i], int(toks[i + 1]), int(toks[i + 2])
            i += 3
            ext = [float(t) for t in toks[i:i + 2 * ndims]]
            i += 2 * ndims
            vel = [0.0, 0.0]
            if bt in ("slip-wall", "noslip-wall"):
                vel = [float(t) for t in toks[i:i + ndims]] + [0.0]
                i += ndims
            P.bc_type[n] = {"periodic": 0, "extrapolate": 1, "slip-wall": 2}[bt]
            P.bc_dim[n], P.bc_face[n] = dim, face
            for d in range(ndims):
                if d == dim:
                    if face == 1:
                        P.bc_is[n][d], P.bc_ie[n][d] = -g, 0
                    else:
                        P.bc_is[n][d], P.bc_ie[n][d] = dims[d], dims[d] + g
                else:
                    is_, ie_ = _find_interval(ext[2 * d], ext[2 * d + 1], xs[d])
                    P.bc_is[n][d], P.bc_ie[n][d] = is_, ie_
            P.bc_vel[n][0], P.bc_vel[n][1] = vel[0], vel[1] if ndims == 2 else 0.0
        self.P = P

    def _ghost_x(self, xi):
        g, N = self.ghosts, len(xi)
        X = np.zeros(N + 2 * g)
        X[g:g + N] = xi
        for i in range(g):
            delta = g - i
            X[i] = X[g] + float(delta) * (X[g] - X[g + 1])
        for i in range(N + g, N + 2 * g):
            delta = i - (N + g - 1)
            X[i] = X[N + g - 1] + float(delta) * (X[N + g - 1] - X[N + g - 2])
        return X

    def _dxinv(self, X, N):
        g = self.ghosts
        d = np.zeros(N + 2 * g)
        for i in range(N):
            d[i + g] = 2.0 / (X[i + 1 + g] - X[i - 1 + g])
        for i in range(g):
            d[i] = d[g]
        for i in range(N + g, N + 2 * g):
            d[i] = d[N + g - 1]
        return d

    def _chemistry(self, path, nflow):
        """ChemistryInitialize.c:69-481: defaults, chemistry.inp, normalisation."""
        ch = dict(pi=4.0 * math.atan(1.0), NA=6.02214076e23, kB=1.380649e-23, c=3.0e8,
                  h=6.62607015e-34, e=1.60217663e-19, M_O2=0.032, M_CO2=0.044,
                  Cp_O2=918.45, Cv_O2=650.0, Cp_CO2=842.86, Cv_CO2=654.5,
                  mu0_O2=1.99e-5, kappa0_O2=2.70e-2, mu0_CO2=1.45e-5, kappa0_CO2=1.58e-2,
                  lambda_UV=2.48e-7, f_CO2=0.0, f_O3=0.005, Ptot=101325.0, Ti=288.0,
                  t_start=0.0, t_pulse=10 * 1e-9, Lz=0.03, z_mm=0.0, nz_layers=22,
                  k0a=0.9 * 3.3e-13, k0b=0.1 * 3.3e-13, k1a=0.8 * 3.95e-17, k1b=0.2 * 3.95e-17,
                  k2a=1.2e-16, k2b=1.2e-16, k3a=1.2e-17, k3b=1.0e-17, k4=1.1e-16, k5=2.0e-16,
                  k6=0.2 * 3.0e-17, F0=2000.0, sO3=1.1e-21, IA=1.0, IB=1.0, IC=0.0)
        ch["theta"] = 0.17 * ch["pi"] / 180
        f = _keyfile(os.path.join(path, "chemistry.inp")) or {}
        keys = {"lambda_UV", "t_start", "t_pulse", "theta", "f_CO2", "f_O3", "Ptot", "Ti", "Lz",
                "z_mm", "k0a", "k1a", "k2a", "k3a", "k0b", "k1b", "k2b", "k3b", "k4", "k5", "k6",
                "F0", "sO3", "IA", "IB", "IC"}
        for k, v in f.items():
            if k == "nz":
                ch["nz_layers"] = int(v)
            elif k in keys:
                ch[k] = float(v)
        ch["f_O2"] = 1.0 - ch["f_CO2"]
        ch["R"] = ch["NA"] * ch["kB"] / (ch["f_O2"] * ch["M_O2"] + ch["f_CO2"] * ch["M_CO2"])
        ch["Cp"] = ch["f_O2"] * ch["Cp_O2"] + ch["f_CO2"] * ch["Cp_CO2"]
        ch["Cv"] = ch["f_O2"] * ch["Cv_O2"] + ch["f_CO2"] * ch["Cv_CO2"]
        ch["gamma"] = ch["Cp"] / ch["Cv"]
        ch["mu0"] = ch["f_O2"] * ch["mu0_O2"] + ch["f_CO2"] * ch["mu0_CO2"]
        ch["kappa0"] = ch["f_O2"] * ch["kappa0_O2"] + ch["f_CO2"] * ch["kappa0_CO2"]
        ch["kUV"] = 2 * ch["pi"] / ch["lambda_UV"]
        ch["kg"] = 2 * ch["kUV"] * math.sin(ch["theta"])
        ch["n_O2"] = ch["f_O2"] * ch["Ptot"] / (ch["kB"] * ch["Ti"])
        ch["n_O3"] = ch["f_O3"] * ch["Ptot"] / (ch["kB"] * ch["Ti"])
        ch["n_CO2"] = ch["f_CO2"] * ch["Ptot"] / (ch["kB"] * ch["Ti"])
        ch["cs"] = math.sqrt(ch["gamma"] * ch["R"] * ch["Ti"])
        ch["L_ref"] = 1.0 / ch["kg"]
        ch["v_ref"] = ch["cs"]
        ch["t_ref"] = ch["L_ref"] / ch["v_ref"]
        ch["rho_ref"] = ch["Ptot"] / (ch["R"] * ch["Ti"])
        ch["P_ref"] = ch["rho_ref"] * ch["v_ref"] * ch["v_ref"]
        ch["t_start_norm"] = ch["t_start"] / ch["t_ref"]
        ch["t_pulse_norm"] = ch["t_pulse"] / ch["t_ref"]
        rate_norm_fac = ch["kg"] * ch["cs"] / ch["n_O2"]
        for k in ["k0a", "k1a", "k2a", "k3a", "k0b", "k1b", "k2b", "k3b", "k4", "k5", "k6"]:
            ch[k + "_norm"] = ch[k] / rate_norm_fac
        ch["I0"] = ch["F0"] / ch["t_pulse"]
        ch["nu"] = ch["c"] / ch["lambda_UV"]
        Ei = ch["P_ref"] / ((ch["gamma"] - 1.0) * ch["n_O2"])
        for k, fac in [("q0a", 0.73), ("q0b", 2.8), ("q1a", 0.29), ("q1b", 0.84), ("q2a", 4.3),
                       ("q2b", 0.81), ("q3a", 0.42), ("q3b", 1.16), ("q4", 1.23), ("q5", 1.81),
                       ("q6", 0.42)]:
            ch[k + "_norm"] = fac * ch["e"] / Ei
        ch["dz"] = ch["Lz"] / ch["nz_layers"]
        ch["z_i"] = int(math.ceil(ch["z_mm"] * 0.001 * ch["nz_layers"] / ch["Lz"]))
        ch["nz"] = ch["z_i"] + 1
        return ch

    # ------------------------------------------------------------- running
    def run(self, nsteps=None, u=None, t0=0.0):
        """Advance ``nsteps`` (default n_iter) RK steps; returns ghosted AoS u."""
        u = (self.u0 if u is None else u).copy()
        n = self.n_iter if nsteps is None else nsteps
        ret = lib().orc_run(C.byref(self.P), _dp(u), _dp(self.dxinv), _dp(self.imap), float(t0), int(n))
        if ret != 0:
            raise RuntimeError("oracle: zero pivot in a tridiagonal solve")
        return u

    def rhs(self, u, t=0.0):
        u = u.copy()
        r = np.zeros_like(u)
        lib().orc_rhs(C.byref(self.P), _dp(r), _dp(u), _dp(self.dxinv), _dp(self.imap), float(t))
        return r, u

    def interior(self, u):
        """AoS ghosted -> (npoints, nvars) interior, dim0 fastest (op-file order)."""
        g = self.ghosts
        a = u.reshape(self.shape_g[0], self.shape_g[1], self.nvars)
        if self.ndims == 2:
            a = a[g:g + self.dims[1], g:g + self.dims[0], :]
        else:
            a = a[0, g:g + self.dims[0], :]
        return np.ascontiguousarray(a.reshape(-1, self.nvars))

    def cfl(self, u):
        return lib().orc_cfl(C.byref(self.P), _dp(u), _dp(self.dxinv))


def load(path: str) -> Case:
    return Case(path)
