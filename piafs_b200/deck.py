"""Reader/writer for the PIAFS input deck and binary output files.

The formats are the reference's contract, restated here so that the GPU path
consumes and produces exactly the files the CPU code does:

* ``solver.inp`` / ``physics.inp`` / ``chemistry.inp`` / ``weno.inp``:
  whitespace ``begin <key> <value>... end`` files
  (src/Simulation/ReadInputs.c:244-450, NavierStokes2DInitialize.c:52-64,
  ChemistryInitialize.c:34-64, WENOInitialize.c:46-90).
* ``boundary.inp``: zone count, then per zone ``type dim face`` followed by
  ``xmin xmax`` for each dimension and type-specific extras (wall velocity for
  slip walls) (src/Simulation/InitializeBoundaries.c:82-150).
* ``initial.inp`` / ``imap.inp`` (binary): the grid coordinates of each
  dimension, then the field with the variable index fastest, then dim0, dim1
  (src/IOFunctions/ReadArray.c:228-257).
* ``op_<nnnnn>.bin``: int32 ndims, int32 nvars, int32 size[ndims], f64 grid,
  f64 field in the same point-major order (src/IOFunctions/WriteBinary.c:37-93).
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np


def _num(v) -> str:
    """A value as the reference's fscanf reads it: floats (numpy ones too) in
    shortest round-trip form, integers plainly, anything else as str."""
    if isinstance(v, (bool, np.bool_)):
        return str(v)
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    if isinstance(v, (float, np.floating)):
        return repr(float(v))
    return str(v)


def write_keyfile(path: str, items: Dict[str, object]) -> None:
    """Write a ``begin ... end`` keyword file, one ``key value`` per line."""
    with open(path, "w") as f:
        f.write("begin\n")
        for k, v in items.items():
            if isinstance(v, (list, tuple)):
                v = " ".join(_num(a) for a in v)
            else:
                v = _num(v)
            f.write(f"  {k:<20s} {v}\n")
        f.write("end\n")


def read_keyfile(path: str) -> Dict[str, List[str]]:
    """Read a ``begin ... end`` keyword file into ``{key: [tokens]}``.

    Tokens are whitespace separated, as the reference's fscanf loop reads them.
    Multi-valued keys (``size``) keep all their tokens.
    """
    with open(path) as f:
        toks = f.read().split()
    if not toks or toks[0] != "begin":
        raise ValueError(f"{path}: illegal format (no 'begin')")
    out: Dict[str, List[str]] = {}
    i = 1
    while i < len(toks) and toks[i] != "end":
        k = toks[i]
        i += 1
        vals = []
        if k in _MULTI_KEYS:
            # numeric list (one value per dimension)
            while i < len(toks) and toks[i] != "end" and _is_number(toks[i]):
                vals.append(toks[i])
                i += 1
        elif i < len(toks):
            vals.append(toks[i])
            i += 1
        out[k] = vals
    return out


_MULTI_KEYS = {"size", "size_exact", "iproc"}


def _is_number(tok: str) -> bool:
    try:
        float(tok)
        return True
    except ValueError:
        return False




@dataclass
class BoundaryZone:
    """One boundary zone of ``boundary.inp``."""
    bctype: str
    dim: int
    face: int
    extent: Sequence[float]            # xmin, xmax for each dimension
    wall_velocity: Optional[Sequence[float]] = None   # slip-wall / noslip-wall
    # the zone's data in the order the reference reads it
    # (InitializeBoundaries.c:106-168): dirichlet / sponge one value per
    # variable; subsonic-inflow density, velocity, passive scalars;
    # subsonic-outflow pressure; subsonic-ambivalent density, velocity,
    # pressure; supersonic-inflow density, velocity, pressure, passive scalars
    values: Optional[Sequence[float]] = None


def write_boundary(path: str, zones: Sequence[BoundaryZone]) -> None:
    with open(path, "w") as f:
        f.write(f"{len(zones)}\n")
        for z in zones:
            ext = " ".join(f"{v:g}" for v in z.extent)
            line = f"{z.bctype:<12s} {z.dim:d} {z.face:2d}  {ext}"
            f.write(line + "\n")
            if z.wall_velocity is not None:
                f.write("  " + " ".join(repr(float(v)) for v in z.wall_velocity) + "\n")
            if z.values is not None:
                f.write("  " + " ".join(repr(float(v)) for v in z.values) + "\n")


def _zone_value_count(bctype: str, ndims: int, nvars: int) -> int:
    nscalars = nvars - (2 + ndims)
    return {"dirichlet": nvars, "sponge": nvars, "subsonic-inflow": 1 + ndims + nscalars,
            "subsonic-outflow": 1, "subsonic-ambivalent": 2 + ndims,
            "supersonic-inflow": 2 + ndims + nscalars}.get(bctype, 0)


def read_boundary(path: str, ndims: int, nvars: int = 0) -> List[BoundaryZone]:
    """Read ``boundary.inp``; ``nvars`` is needed for the zone types whose data
    depends on it (dirichlet, sponge and the inflows with passive scalars)."""
    toks = open(path).read().split()
    n = int(toks[0])
    i = 1
    zones = []
    for _ in range(n):
        bctype, dim, face = toks[i], int(toks[i + 1]), int(toks[i + 2])
        i += 3
        ext = [float(t) for t in toks[i:i + 2 * ndims]]
        i += 2 * ndims
        wv = None
        if bctype in ("slip-wall", "noslip-wall"):
            wv = [float(t) for t in toks[i:i + ndims]]
            i += ndims
        nval = _zone_value_count(bctype, ndims, nvars)
        vals = [float(t) for t in toks[i:i + nval]] if nval else None
        i += nval
        zones.append(BoundaryZone(bctype, dim, face, ext, wv, vals))
    return zones


def write_array_binary(path: str, grid: Sequence[np.ndarray], field_pm: np.ndarray) -> None:
    """Write ``initial.inp``-style binary: grids then point-major field.

    ``field_pm`` has shape ``(npoints, nvars)`` with dim0 fastest in the point
    index (ReadArray.c:228-257).
    """
    with open(path, "wb") as f:
        for g in grid:
            np.asarray(g, dtype=np.float64).tofile(f)
        np.ascontiguousarray(field_pm, dtype=np.float64).tofile(f)


def read_array_binary(path: str, dims: Sequence[int], nvars: int):
    with open(path, "rb") as f:
        grids = [np.fromfile(f, dtype=np.float64, count=d) for d in dims]
        npts = int(np.prod(dims))
        u = np.fromfile(f, dtype=np.float64, count=npts * nvars)
    if u.size != npts * nvars:
        raise ValueError(f"{path}: short read ({u.size} of {npts * nvars} values)")
    return grids, u.reshape(npts, nvars)


@dataclass
class OpFile:
    ndims: int
    nvars: int
    size: np.ndarray
    grid: List[np.ndarray]
    u: np.ndarray               # (npoints, nvars), dim0 fastest


def read_op(path: str) -> OpFile:
    """Read an ``op_*.bin`` written by WriteBinary (WriteBinary.c:37-93)."""
    with open(path, "rb") as f:
        ndims = int(np.fromfile(f, dtype=np.int32, count=1)[0])
        nvars = int(np.fromfile(f, dtype=np.int32, count=1)[0])
        size = np.fromfile(f, dtype=np.int32, count=ndims)
        grid = [np.fromfile(f, dtype=np.float64, count=int(s)) for s in size]
        npts = int(np.prod(size))
        u = np.fromfile(f, dtype=np.float64, count=npts * nvars)
    return OpFile(ndims, nvars, size, grid, u.reshape(npts, nvars))


def write_op(path: str, grid: Sequence[np.ndarray], u_pm: np.ndarray) -> None:
    """Write an ``op_*.bin`` in the reference's binary layout."""
    ndims = len(grid)
    nvars = u_pm.shape[1]
    with open(path, "wb") as f:
        np.array([ndims, nvars], dtype=np.int32).tofile(f)
        np.array([len(g) for g in grid], dtype=np.int32).tofile(f)
        for g in grid:
            np.asarray(g, dtype=np.float64).tofile(f)
        np.ascontiguousarray(u_pm, dtype=np.float64).tofile(f)


def op_filename(index: int, root: str = "op", ext: str = ".bin") -> str:
    """``op_00000.bin`` style name: 5-digit zero-padded index
    (InitializeSolvers.c:219-222, WriteArray.c:133-139)."""
    return f"{root}_{index:05d}{ext}"


def rel_norms(u: np.ndarray, ref: np.ndarray, per_var: bool = True):
    """Relative L1/L2/Linf error norms, CompareSolutions-style.

    Follows Extras/CompareSolutions.c:812-906: L1 = sum|d|/N, L2 =
    sqrt(sum d^2/N), Linf = max|d|, each divided by the same norm of the
    reference unless that norm is <= 1e-15, in which case the absolute norm is
    reported.  ``per_var`` applies it to each conserved variable separately
    (u, ref of shape (npoints, nvars)); otherwise to all variables together.
    """
    u = np.asarray(u, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if u.shape != ref.shape:
        raise ValueError(f"shape mismatch {u.shape} vs {ref.shape}")

    def one(a, r):
        d = a - r
        n = a.size
        l1, l2, li = np.abs(d).sum() / n, np.sqrt((d * d).sum() / n), np.abs(d).max()
        r1, r2, ri = np.abs(r).sum() / n, np.sqrt((r * r).sum() / n), np.abs(r).max()
        return (l1 / r1 if r1 > 1e-15 else l1,
                l2 / r2 if r2 > 1e-15 else l2,
                li / ri if ri > 1e-15 else li)

    if not per_var:
        return one(u.ravel(), ref.ravel())
    return [one(u[:, v], ref[:, v]) for v in range(u.shape[1])]
