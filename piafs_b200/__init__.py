"""piafs_b200 -- B200 (sm_100a) implementation of PIAFS's per-stage
right-hand side and explicit Runge-Kutta time step.

The compute path is the native library ``libpiafs_gpu.so`` (hand-written CUDA
kernels behind the C ABI of ``include/piafs_gpu.h``); this module is a thin
ctypes host binding.  It mirrors the reference's simulation flow
(ReadInputs/Initialize -> Solve, src/main.cpp:68-247) and the HyPar operator
function pointers (include/hypar.h:204-290):

    sim = Simulation("path/to/deck")     # the reference's input deck
    sim.solve("path/to/deck")            # op_NNNNN.bin like the CPU code
    sim.time_rk(10)                      # TimeIntegrate, device-resident
    u = sim.solution()                   # (npoints, nvars), output order

Operator-level calls take CUDA device pointers (or torch CUDA tensors) in the
reference's array-of-structures layout.  There is no CPU fallback: if the
library or a CUDA device is missing, these calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import cases, deck  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpiafs_gpu.so")
CLI_PATH = os.path.join(HERE, "bin", "piafs-gpu")

PIAFS_OK = 0
ERRORS = {1: "argument", 2: "input", 3: "unsupported", 4: "cuda", 5: "singular", 6: "io", 7: "memory"}
PRECISION = {"fp64": 0, "mixed": 1}

# Every entry point of include/piafs_gpu.h with its ctypes signature.
_dp = C.POINTER(C.c_double)
_vp = C.c_void_p
SIGNATURES = {
    "piafs_gpu_last_error": (C.c_char_p, []),
    "piafs_gpu_create": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(_vp)]),
    "piafs_gpu_destroy": (None, [_vp]),
    "piafs_gpu_get_info": (C.c_int, [_vp, _vp]),
    "piafs_gpu_set_state": (C.c_int, [_vp, _dp, C.c_double]),
    "piafs_gpu_get_state": (C.c_int, [_vp, _dp]),
    "piafs_gpu_get_solution": (C.c_int, [_vp, _dp]),
    "piafs_gpu_TimeRK": (C.c_int, [_vp, C.c_int]),
    "piafs_gpu_TimeRK_norm": (C.c_int, [_vp, C.c_int, _dp]),
    "piafs_gpu_WriteErrors": (C.c_int, [_vp, C.c_char_p, C.c_double, C.c_double]),
    "piafs_gpu_get_photon_density": (C.c_int, [_vp, _dp]),
    "piafs_gpu_TimeRK_host": (C.c_int, [_vp, _dp, C.c_double]),
    "piafs_gpu_Solve": (C.c_int, [_vp, C.c_char_p]),
    "piafs_gpu_ComputeCFL": (C.c_int, [_vp, _dp]),
    "piafs_gpu_TimeRK_async": (C.c_int, [_vp, C.c_int]),
    "piafs_gpu_get_stream": (C.c_int, [_vp, C.POINTER(_vp)]),
    "piafs_gpu_synchronize": (C.c_int, [_vp]),
    "piafs_gpu_profile_rhs": (C.c_int, [_vp, C.c_int, _dp, C.POINTER(C.c_int)]),
    "piafs_gpu_RHSFunction": (C.c_int, [_vp, _vp, _vp, C.c_double]),
    "piafs_gpu_HyperbolicFunction": (C.c_int, [_vp, _vp, _vp, C.c_double]),
    "piafs_gpu_ParabolicFunction": (C.c_int, [_vp, _vp, _vp, C.c_double]),
    "piafs_gpu_SourceFunction": (C.c_int, [_vp, _vp, _vp, C.c_double]),
    "piafs_gpu_ApplyBoundaryConditions": (C.c_int, [_vp, _vp, C.c_double]),
    "piafs_gpu_FFunction": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_double]),
    "piafs_gpu_InterpolateInterfacesHyp": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_int, C.c_int]),
    "piafs_gpu_Upwind": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, C.c_int, C.c_double]),
    "piafs_gpu_FirstDerivativePar": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, C.c_int]),
    "piafs_gpu_tridiagLU": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_int]),
    "piafs_gpu_HyperbolicFunction_noalloc": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "piafs_gpu_reciprocal": (C.c_int, [_vp, _vp, C.c_longlong]),
    "piafs_gpu_batch_create": (C.c_int, [C.c_int, C.c_ulonglong, C.POINTER(C.c_void_p)]),
    "piafs_gpu_batch_destroy": (None, [_vp]),
    "piafs_gpu_batch_add": (C.c_int, [_vp, C.c_char_p, C.c_int, C.POINTER(C.c_int)]),
    "piafs_gpu_batch_step": (C.c_int, [_vp, C.c_int]),
    "piafs_gpu_batch_add_many": (C.c_int, [_vp, C.POINTER(C.c_char_p), C.c_int, C.POINTER(C.c_int),
                                           C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "piafs_gpu_batch_poll": (C.c_int, [_vp, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]),
    "piafs_gpu_batch_get_solution": (C.c_int, [_vp, C.c_int, _dp]),
    "piafs_gpu_batch_member": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int),
                                         C.POINTER(C.c_int)]),
    "piafs_gpu_batch_remove": (C.c_int, [_vp, C.c_int]),
    "piafs_gpu_batch_get_stage_derivative": (C.c_int, [_vp, C.c_int, C.c_int, _dp]),
    "piafs_gpu_batch_get_buffer": (C.c_int, [_vp, C.c_int, C.c_int, _dp]),
    "piafs_gpu_batch_get_info": (C.c_int, [_vp, _vp]),
    "piafs_gpu_batch_tune": (C.c_int, [_vp, C.c_int]),
    "piafs_gpu_batch_set_launch": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int]),
    "piafs_gpu_batch_add_request": (C.c_int, [_vp, _vp, C.POINTER(C.c_int)]),
    "piafs_gpu_batch_checksum": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_double)]),
    "piafs_gpu_serve_trace": (C.c_int, [_vp, _vp, C.c_int, C.c_int, C.c_ulonglong, C.c_ulonglong, C.c_int, _vp]),
    "piafs_gpu_slab_create": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(_vp)]),
    "piafs_gpu_slab_destroy": (None, [_vp]),
    "piafs_gpu_slab_get_info": (C.c_int, [_vp, _vp]),
    "piafs_gpu_slab_sim": (C.c_int, [_vp, C.POINTER(_vp)]),
    "piafs_gpu_slab_state": (C.c_int, [_vp, C.c_int, C.POINTER(_vp)]),
    "piafs_gpu_slab_buffers": (C.c_int, [_vp, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(_vp)]),
    "piafs_gpu_slab_stage_begin": (C.c_int, [_vp, C.c_int]),
    "piafs_gpu_slab_y_pass": (C.c_int, [_vp, C.c_int]),
    "piafs_gpu_slab_stage_end": (C.c_int, [_vp, C.c_int]),
    "piafs_gpu_slab_step_end": (C.c_int, [_vp, C.c_int]),
    "piafs_gpu_slab_norm_sum": (C.c_int, [_vp, _dp]),
}


class HypParams(C.Structure):
    """piafs_gpu_hyp_params of include/piafs_gpu.h."""
    _fields_ = [
        ("ndims", C.c_int), ("nvars", C.c_int), ("ghosts", C.c_int), ("dim", C.c_int * 2),
        ("model", C.c_int), ("scheme", C.c_int), ("upwind", C.c_int), ("weno_type", C.c_int),
        ("no_limiting", C.c_int), ("weno_eps", C.c_double), ("gamma", C.c_double),
    ]


class Info(C.Structure):
    _fields_ = [
        ("ndims", C.c_int), ("nvars", C.c_int), ("ghosts", C.c_int), ("dim", C.c_int * 2),
        ("n_iter", C.c_int), ("restart_iter", C.c_int), ("screen_op_iter", C.c_int),
        ("file_op_iter", C.c_int), ("iter", C.c_int), ("nstages", C.c_int),
        ("dt", C.c_double), ("t", C.c_double), ("gamma", C.c_double), ("Re", C.c_double),
        ("Pr", C.c_double), ("npoints_ghosted", C.c_longlong), ("ninterfaces", C.c_longlong * 2),
        ("cfl", C.c_double), ("norm", C.c_double), ("singular", C.c_int),
        ("launches_per_step", C.c_int),
    ]

    def asdict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


class PiafsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"piafs_gpu error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libpiafs_gpu.so (building it first if this is a source tree with
    nvcc but no library).  Raises if it cannot be had: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        from . import build as _build
        _build.build()
    L = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _check(code: int):
    if code != PIAFS_OK:
        raise PiafsError(code, _lib.piafs_gpu_last_error().decode())


def _ptr(x) -> int:
    """Device pointer of a torch CUDA tensor, or an int pointer as is."""
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if not x.is_cuda or x.dtype.__str__() != "torch.float64" or not x.is_contiguous():
            raise ValueError("expected a contiguous float64 CUDA tensor")
        return x.data_ptr()
    raise TypeError(f"cannot take a device pointer of {type(x)}")


def _hp(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise ValueError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_dp)


class Simulation:
    """One PIAFS simulation resident on the current CUDA device."""

    def __init__(self, deck_dir: str, precision: str = "fp64"):
        L = load_library()
        h = _vp()
        _check(L.piafs_gpu_create(os.fsencode(deck_dir), PRECISION[precision], C.byref(h)))
        self._h = h
        self.deck_dir = deck_dir

    def close(self):
        if getattr(self, "_h", None):
            _lib.piafs_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---------------------------------------------------------------- info
    @property
    def info(self) -> dict:
        inf = Info()
        _check(_lib.piafs_gpu_get_info(self._h, C.byref(inf)))
        return inf.asdict()

    @property
    def shape_ghosted(self):
        i = self.info
        return (i["npoints_ghosted"], i["nvars"])

    @property
    def shape_interior(self):
        i = self.info
        return (i["dim"][0] * i["dim"][1], i["nvars"])

    # --------------------------------------------------------------- state
    def set_state(self, u: np.ndarray, t: float = 0.0):
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.size != int(np.prod(self.shape_ghosted)):
            raise ValueError("state must be a ghosted array in the reference layout")
        _check(_lib.piafs_gpu_set_state(self._h, _hp(u), float(t)))

    def state(self) -> np.ndarray:
        u = np.empty(self.shape_ghosted)
        _check(_lib.piafs_gpu_get_state(self._h, _hp(u)))
        return u.reshape(-1)

    def solution(self) -> np.ndarray:
        u = np.empty(self.shape_interior)
        _check(_lib.piafs_gpu_get_solution(self._h, _hp(u)))
        return u

    # ------------------------------------------------------------ stepping
    def time_rk(self, nsteps: int = 1):
        """TimeIntegrate on the device-resident state (TimeRK.c:34)."""
        _check(_lib.piafs_gpu_TimeRK(self._h, int(nsteps)))

    def time_rk_norm(self, nsteps: int = 1) -> float:
        """Advance nsteps steps; the residual norm of the last one
        (TimePostStep.c:36-54)."""
        n = C.c_double()
        _check(_lib.piafs_gpu_TimeRK_norm(self._h, int(nsteps), C.byref(n)))
        return n.value

    def write_errors(self, directory: str, solver_runtime: float = 0.0, main_runtime: float = 0.0):
        """errors.dat, conservation.dat and function_counts.dat in directory
        (SimulationWriteErrors.c:65-80)."""
        _check(_lib.piafs_gpu_WriteErrors(self._h, os.fsencode(directory), float(solver_runtime),
                                          float(main_runtime)))

    def time_rk_host(self, u: np.ndarray, t: float) -> np.ndarray:
        """One step on a host array in the reference layout, in place."""
        _check(_lib.piafs_gpu_TimeRK_host(self._h, _hp(u), float(t)))
        return u

    def time_rk_async(self, nsteps: int = 1):
        """Enqueue nsteps steps on the simulation's stream without waiting."""
        _check(_lib.piafs_gpu_TimeRK_async(self._h, int(nsteps)))

    def synchronize(self):
        _check(_lib.piafs_gpu_synchronize(self._h))

    @property
    def stream(self) -> int:
        """The simulation's cudaStream_t as an integer handle."""
        p = _vp()
        _check(_lib.piafs_gpu_get_stream(self._h, C.byref(p)))
        return p.value or 0

    def profile_rhs(self, reps: int = 3):
        """Per-phase device time (ms) of one RHS evaluation (see piafs_gpu.h)."""
        ms = (C.c_double * 16)()
        n = C.c_int(16)
        _check(_lib.piafs_gpu_profile_rhs(self._h, int(reps), ms, C.byref(n)))
        names = []
        for d in range(self.info["ndims"]):
            names += [f"flux_{'xy'[d]}", f"reconstruct_{'xy'[d]}"]
        names += ["upwind_div", "viscous_source"]
        return dict(zip(names, list(ms)[: n.value]))

    def solve(self, output_dir: Optional[str] = None):
        """The reference's Solve() loop with op_NNNNN.bin output."""
        _check(_lib.piafs_gpu_Solve(self._h, os.fsencode(output_dir or self.deck_dir)))

    def cfl(self) -> float:
        c = C.c_double()
        _check(_lib.piafs_gpu_ComputeCFL(self._h, C.byref(c)))
        return c.value

    # ------------------------------------------------ operator-level calls
    def RHSFunction(self, rhs, u, t=0.0):
        _check(_lib.piafs_gpu_RHSFunction(self._h, _ptr(rhs), _ptr(u), float(t)))

    def HyperbolicFunction(self, hyp, u, t=0.0):
        _check(_lib.piafs_gpu_HyperbolicFunction(self._h, _ptr(hyp), _ptr(u), float(t)))

    def ParabolicFunction(self, par, u, t=0.0):
        _check(_lib.piafs_gpu_ParabolicFunction(self._h, _ptr(par), _ptr(u), float(t)))

    def SourceFunction(self, src, u, t=0.0):
        _check(_lib.piafs_gpu_SourceFunction(self._h, _ptr(src), _ptr(u), float(t)))

    def ApplyBoundaryConditions(self, u, t=0.0):
        _check(_lib.piafs_gpu_ApplyBoundaryConditions(self._h, _ptr(u), float(t)))

    def FFunction(self, f, u, dir, t=0.0):
        _check(_lib.piafs_gpu_FFunction(self._h, _ptr(f), _ptr(u), int(dir), float(t)))

    def InterpolateInterfacesHyp(self, fI, fC, u, upw, dir, uflag):
        _check(_lib.piafs_gpu_InterpolateInterfacesHyp(self._h, _ptr(fI), _ptr(fC), _ptr(u), int(upw), int(dir),
                                                       int(uflag)))

    def Upwind(self, fI, fL, fR, uL, uR, u, dir, t=0.0):
        _check(_lib.piafs_gpu_Upwind(self._h, _ptr(fI), _ptr(fL), _ptr(fR), _ptr(uL), _ptr(uR), _ptr(u), int(dir),
                                     float(t)))

    def FirstDerivativePar(self, Df, f, dir, bias, nv):
        _check(_lib.piafs_gpu_FirstDerivativePar(self._h, _ptr(Df), _ptr(f), int(dir), int(bias), int(nv)))


def hyperbolic_noalloc(params: "HypParams", hyp, u, dxinv, stream: int = 0):
    """Allocation-free hyperbolic term (piafs_gpu_HyperbolicFunction_noalloc)."""
    L = load_library()
    code = L.piafs_gpu_HyperbolicFunction_noalloc(C.byref(params), _ptr(hyp), _ptr(u), _ptr(dxinv), stream)
    if code != PIAFS_OK:
        raise PiafsError(code, L.piafs_gpu_last_error().decode())


REQUEST_EULER1D_WAVE, REQUEST_NS2D_BEAM = 1, 2


class Request(C.Structure):
    """A parameter-described solve (piafs_gpu_request)."""
    _fields_ = [
        ("kind", C.c_int), ("n", C.c_int), ("nsteps", C.c_int), ("dt", C.c_double), ("amp", C.c_double),
        ("beam_radius", C.c_double), ("Re", C.c_double), ("noise", C.c_double), ("seed", C.c_ulonglong),
    ]


class ServeResult(C.Structure):
    _fields_ = [("arrival_s", C.c_double), ("admitted_s", C.c_double), ("finished_s", C.c_double),
                ("steps", C.c_int), ("checksum", C.c_double)]


def serve_trace(requests, arrivals, precision: str = "fp64", hbm_budget_bytes: int = 0, steps_per_round: int = 4,
                max_resident_points: int = 0):
    """Replay a request trace in real time through the continuous-batching
    serving loop (piafs_gpu_serve_trace); returns a list of dicts per request
    (arrival, admission, finish in seconds from the start, steps, checksum).
    max_resident_points bounds the grid points resident at once (0: only the
    HBM budget bounds admission)."""
    L = load_library()
    n = len(requests)
    reqs = (Request * n)(*requests)
    arr = (C.c_double * n)(*[float(x) for x in arrivals])
    out = (ServeResult * n)()
    code = L.piafs_gpu_serve_trace(reqs, arr, n, PRECISION[precision], int(hbm_budget_bytes),
                                   int(max_resident_points), int(steps_per_round), out)
    if code != PIAFS_OK:
        raise PiafsError(code, L.piafs_gpu_last_error().decode())
    return [{name: getattr(r, name) for name, _ in ServeResult._fields_} for r in out]


class BatchInfo(C.Structure):
    _fields_ = [
        ("members", C.c_int), ("active", C.c_int), ("tiles", C.c_int), ("tile_x", C.c_int),
        ("tile_y", C.c_int), ("steps", C.c_longlong), ("bytes_in_use", C.c_ulonglong),
        ("budget_bytes", C.c_ulonglong), ("launches_per_step", C.c_int), ("min_ctas_per_sm", C.c_int),
    ]

    def asdict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class Batch:
    """Many independent simulations resident on the device and advanced
    together by one persistent kernel per RK stage (piafs_gpu_batch_*)."""

    def __init__(self, precision: str = "fp64", hbm_budget_bytes: int = 0):
        L = load_library()
        h = _vp()
        _check(L.piafs_gpu_batch_create(PRECISION[precision], int(hbm_budget_bytes), C.byref(h)))
        self._h = h
        self._shapes = {}

    def close(self):
        if getattr(self, "_h", None):
            _lib.piafs_gpu_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def add(self, deck_dir: str, nsteps: int = 0) -> int:
        """Admit a member; raises PiafsError (code PIAFS_ERR_MEMORY when the
        budget cannot hold it now)."""
        i = C.c_int()
        _check(_lib.piafs_gpu_batch_add(self._h, os.fsencode(deck_dir), int(nsteps), C.byref(i)))
        d = deck.read_keyfile(os.path.join(deck_dir, "solver.inp"))
        size = [int(x) for x in d["size"]]
        self._shapes[i.value] = (int(np.prod(size)), int(d["nvars"][0]))
        return i.value

    def add_many(self, deck_dirs, nsteps=None) -> list:
        """Admit many members; decks are parsed in parallel host threads."""
        n = len(deck_dirs)
        dirs = (C.c_char_p * n)(*[os.fsencode(d) for d in deck_dirs])
        steps = (C.c_int * n)(*[int(x) for x in nsteps]) if nsteps is not None else None
        ids = (C.c_int * n)()
        added = C.c_int()
        code = _lib.piafs_gpu_batch_add_many(self._h, dirs, n, steps, ids, C.byref(added))
        for k in range(added.value):
            d = deck.read_keyfile(os.path.join(deck_dirs[k], "solver.inp"))
            self._shapes[ids[k]] = (int(np.prod([int(x) for x in d["size"]])), int(d["nvars"][0]))
        _check(code)
        return list(ids)

    def add_request(self, req: "Request") -> int:
        i = C.c_int()
        _check(_lib.piafs_gpu_batch_add_request(self._h, C.byref(req), C.byref(i)))
        npts = req.n if req.kind == REQUEST_EULER1D_WAVE else req.n * req.n
        self._shapes[i.value] = (npts, 3 if req.kind == REQUEST_EULER1D_WAVE else 11)
        return i.value

    def checksum(self, member: int) -> float:
        s = C.c_double()
        _check(_lib.piafs_gpu_batch_checksum(self._h, int(member), C.byref(s)))
        return s.value

    def step(self, nsteps: int = 1):
        _check(_lib.piafs_gpu_batch_step(self._h, int(nsteps)))

    def poll(self, cap: int = 4096):
        buf = (C.c_int * cap)()
        n = C.c_int()
        _check(_lib.piafs_gpu_batch_poll(self._h, buf, cap, C.byref(n)))
        return list(buf[: n.value])

    def solution(self, member: int) -> np.ndarray:
        npts, nv = self._shapes[member]
        u = np.empty((npts, nv))
        _check(_lib.piafs_gpu_batch_get_solution(self._h, int(member), _hp(u)))
        return u

    def stage_derivative(self, member: int, stage: int) -> np.ndarray:
        npts, nv = self._shapes[member]
        k = np.empty((npts, nv))
        _check(_lib.piafs_gpu_batch_get_stage_derivative(self._h, int(member), int(stage), _hp(k)))
        return k

    def member(self, member: int) -> dict:
        t, it, done = C.c_double(), C.c_int(), C.c_int()
        _check(_lib.piafs_gpu_batch_member(self._h, int(member), C.byref(t), C.byref(it), C.byref(done)))
        return {"t": t.value, "iter": it.value, "done": bool(done.value)}

    def remove(self, member: int):
        _check(_lib.piafs_gpu_batch_remove(self._h, int(member)))
        self._shapes.pop(member, None)

    @property
    def info(self) -> dict:
        inf = BatchInfo()
        _check(_lib.piafs_gpu_batch_get_info(self._h, C.byref(inf)))
        return inf.asdict()

    def tune(self, tile_x: int = 0):
        """Autotune the launch configuration on the current members (tile_x =
        0), or force a tile width."""
        _check(_lib.piafs_gpu_batch_tune(self._h, int(tile_x)))

    def set_launch(self, tile_x: int, tile_y: int, min_ctas_per_sm: int = 1):
        _check(_lib.piafs_gpu_batch_set_launch(self._h, int(tile_x), int(tile_y), int(min_ctas_per_sm)))


def reciprocal(x, y):
    """y = 1/x on device arrays by the kernels' Newton-Raphson reciprocal."""
    L = load_library()
    code = L.piafs_gpu_reciprocal(_ptr(x), _ptr(y), int(x.numel()))
    if code != PIAFS_OK:
        raise PiafsError(code, L.piafs_gpu_last_error().decode())


def tridiagLU(a, b, c, x, n: int, ns: int):
    """Batched tridiagonal solve, reference layout [row * ns + system]."""
    L = load_library()
    code = L.piafs_gpu_tridiagLU(_ptr(a), _ptr(b), _ptr(c), _ptr(x), int(n), int(ns))
    if code != PIAFS_OK:
        raise PiafsError(code, L.piafs_gpu_last_error().decode())
