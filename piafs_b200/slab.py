"""A 2D grid decomposed along y, one GPU per row slab: the host side of
include/piafs_gpu.h's ``piafs_gpu_slab_*``.

The reference runs one grid on many MPI ranks: each rank owns a block of the
grid, ghost points are exchanged before every right-hand side
(MPIExchangeBoundariesnD.c:45-177), and CRWENO5 systems whose lines cross
ranks are solved by the MPI-parallel tridiagLU (tridiagLU.c:16-85, 155-240).
Here rank r owns the rows [r n1, (r+1) n1) (its row slab, where every x line
is whole) and, for the y direction, the columns [r n0, (r+1) n0) over all
rows (its column slab, where every y line is whole), so every tridiagonal
system is solved whole on one GPU by the same kernel as on an undecomposed
grid.  Per RK stage three exchanges move data between the slabs, each one
all-to-all:

* halo     -- the g rows next to each slab edge to the neighbouring slab's
              ghost rows (around the ends when the grid is periodic in y);
* columns  -- the stage state, ghost rows included, to the column slabs,
              transposed so that y lines are contiguous;
* hy       -- the y term of the hyperbolic divergence back to the row slabs.

``SlabLayout`` holds the index arithmetic on torch tensors of any device
(the CPU tests run it over gloo); ``SlabSimulation`` runs one rank's slab
under torch.distributed (NCCL: one process per GPU, collectives on the
library's stream); ``LocalSlabs`` runs every slab of a grid in one process
and moves the data with copies, which checks the decomposition on one GPU.
Both give the undecomposed simulation's solution bit for bit.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional

import numpy as np

from . import PRECISION, _check, _hp, load_library

_vp = C.c_void_p


class SlabInfo(C.Structure):
    """piafs_gpu_slab_info of include/piafs_gpu.h."""
    _fields_ = [
        ("rank", C.c_int), ("nranks", C.c_int), ("dim", C.c_int * 2), ("slab_rows", C.c_int),
        ("slab_cols", C.c_int), ("ghosts", C.c_int), ("nvars", C.c_int), ("nstages", C.c_int),
        ("periodic_y", C.c_int), ("plane_stride", C.c_longlong), ("col_plane_stride", C.c_longlong),
        ("hy_bytes", C.c_longlong), ("hy_value_bytes", C.c_int),
    ]


def _lib():
    return load_library()


class SlabLayout:
    """Where each exchanged value comes from and goes to.

    Row-slab state: [nvars][plane_stride], the first (n1 + 2g)(N0 + 2g)
    values of a plane being rows -g .. n1+g-1 of the slab, each N0 + 2g wide.
    Column-slab state: [nvars][col_plane_stride], the first
    (n0 + 2g)(N1 + 2g) values of a plane being columns -g .. n0+g-1, each
    N1 + 2g rows long.  The y term: [nranks][nvars][n1][n0] on both sides.
    """

    def __init__(self, N0: int, N1: int, ghosts: int, nvars: int, nranks: int, plane_stride: int,
                 col_plane_stride: int, periodic_y: bool):
        if N0 % nranks or N1 % nranks:
            raise ValueError("grid sides must be multiples of the number of slabs")
        self.N0, self.N1, self.g, self.nvars, self.P = N0, N1, ghosts, nvars, nranks
        self.n0, self.n1 = N0 // nranks, N1 // nranks
        self.ps, self.psc = plane_stride, col_plane_stride
        self.periodic = bool(periodic_y)
        self.W0, self.w1 = N0 + 2 * ghosts, self.n1 + 2 * ghosts
        self.W0c, self.W1c = self.n0 + 2 * ghosts, N1 + 2 * ghosts

    # neighbours along y
    def up(self, r: int) -> Optional[int]:
        return r + 1 if r + 1 < self.P else (0 if self.periodic else None)

    def down(self, r: int) -> Optional[int]:
        return r - 1 if r > 0 else (self.P - 1 if self.periodic else None)

    def rows(self, U):
        """[nvars, n1 + 2g, N0 + 2g] view of a row-slab state."""
        return U.view(self.nvars, self.ps)[:, : self.w1 * self.W0].view(self.nvars, self.w1, self.W0)

    def cols(self, utc):
        """[nvars, n0 + 2g, N1 + 2g] view of a column-slab state."""
        return utc.view(self.nvars, self.psc)[:, : self.W0c * self.W1c].view(self.nvars, self.W0c, self.W1c)

    # ---------------------------------------------------------------- halo
    def _halo_parts(self, r: int, k: int):
        """Which of rank r's edge rows go to rank k, in order: 'top' (its
        last g interior rows, k's lower ghosts) and 'bottom' (its first g
        rows, k's upper ghosts)."""
        parts = []
        if k == self.up(r):
            parts.append("top")
        if k == self.down(r):
            parts.append("bottom")
        return parts

    def halo_send(self, r: int, U):
        """Rank r's send buffer and per-destination sizes (values)."""
        import torch
        V = self.rows(U)
        g, n1 = self.g, self.n1
        blocks, sizes = [], []
        for k in range(self.P):
            bs = []
            for part in self._halo_parts(r, k):
                bs.append((V[:, n1: n1 + g, :] if part == "top" else V[:, g: 2 * g, :]).reshape(-1))
            sizes.append(sum(b.numel() for b in bs))
            blocks.extend(bs)
        send = torch.cat(blocks) if blocks else U.new_empty(0)
        return send, sizes

    def halo_recv_sizes(self, r: int):
        return [len(self._halo_parts(s, r)) * self.nvars * self.g * self.W0 for s in range(self.P)]

    def halo_apply(self, r: int, U, recv):
        """Store what rank r received into its ghost rows."""
        V = self.rows(U)
        g, n1, blk = self.g, self.n1, self.nvars * self.g * self.W0
        off = 0
        for s in range(self.P):
            for part in self._halo_parts(s, r):
                piece = recv[off: off + blk].view(self.nvars, g, self.W0)
                if part == "top":        # the lower neighbour's top rows: my lower ghosts
                    V[:, 0:g, :].copy_(piece)
                else:                    # the upper neighbour's bottom rows: my upper ghosts
                    V[:, n1 + g: n1 + 2 * g, :].copy_(piece)
                off += blk

    # ------------------------------------------------------------- columns
    def column_send(self, U):
        """[nranks, nvars, n0, n1 + 2g]: block c holds columns
        [c n0, (c+1) n0) of every row of the slab (ghost rows included),
        row index fastest."""
        V = self.rows(U)
        g = self.g
        X = V[:, :, g: g + self.N0].reshape(self.nvars, self.w1, self.P, self.n0)
        return X.permute(2, 0, 3, 1).contiguous()

    def column_apply(self, recv, utc):
        """Assemble the column slab from the row slabs' blocks: interior rows
        from every slab, the lower ghost rows from the first, the upper ghost
        rows from the last."""
        g, n1, n0, P = self.g, self.n1, self.n0, self.P
        Cv = self.cols(utc)
        R = recv.view(P, self.nvars, n0, self.w1)
        inner = R[:, :, :, g: g + n1].permute(1, 2, 0, 3).reshape(self.nvars, n0, P * n1)
        Cv[:, g: g + n0, g: g + self.N1].copy_(inner)
        Cv[:, g: g + n0, 0:g].copy_(R[0, :, :, 0:g])
        Cv[:, g: g + n0, g + self.N1: 2 * g + self.N1].copy_(R[P - 1, :, :, g + n1: 2 * g + n1])


# --------------------------------------------------------------------- device
class _DeviceArray:
    """A device pointer as a __cuda_array_interface__ object, so that torch
    sees the library's buffers without copying them."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def _view(ptr: int, n: int, dtype):
    import torch
    typestr = "<f8" if dtype == torch.float64 else "<f4"
    return torch.as_tensor(_DeviceArray(ptr, n, typestr), device="cuda")


class _Slab:
    """One row slab on the current device: library handle and torch views."""

    def __init__(self, deck_dir: str, precision: str, rank: int, nranks: int):
        import torch
        L = _lib()
        self.L = L
        h = _vp()
        _check(L.piafs_gpu_slab_create(os.fsencode(deck_dir), PRECISION[precision], rank, nranks, C.byref(h)))
        self.h = h
        inf = SlabInfo()
        _check(L.piafs_gpu_slab_get_info(h, C.byref(inf)))
        self.info = inf
        self.rank, self.nranks = rank, nranks
        self.layout = SlabLayout(inf.dim[0], inf.dim[1], inf.ghosts, inf.nvars, nranks, inf.plane_stride,
                                 inf.col_plane_stride, bool(inf.periodic_y))
        sim = _vp()
        _check(L.piafs_gpu_slab_sim(h, C.byref(sim)))
        self.sim = sim
        st = _vp()
        _check(L.piafs_gpu_get_stream(sim, C.byref(st)))
        self.stream = st.value or 0
        nv = inf.nvars
        self.U = []
        for k in range(inf.nstages):
            p = _vp()
            _check(L.piafs_gpu_slab_state(h, k, C.byref(p)))
            self.U.append(_view(p.value, nv * inf.plane_stride, torch.float64))
        utc, hs, hr = _vp(), _vp(), _vp()
        _check(L.piafs_gpu_slab_buffers(h, C.byref(utc), C.byref(hs), C.byref(hr)))
        self.utc = _view(utc.value, nv * inf.col_plane_stride, torch.float64)
        hdt = torch.float64 if inf.hy_value_bytes == 8 else torch.float32
        nhy = inf.hy_bytes // inf.hy_value_bytes
        self.hy_send = _view(hs.value, nhy, hdt)
        self.hy_recv = _view(hr.value, nhy, hdt)

    def close(self):
        if getattr(self, "h", None):
            self.L.piafs_gpu_slab_destroy(self.h)
            self.h = None

    def stage_begin(self, st):
        _check(self.L.piafs_gpu_slab_stage_begin(self.h, st))

    def y_pass(self, st):
        _check(self.L.piafs_gpu_slab_y_pass(self.h, st))

    def stage_end(self, st):
        _check(self.L.piafs_gpu_slab_stage_end(self.h, st))

    def step_end(self, with_norm):
        _check(self.L.piafs_gpu_slab_step_end(self.h, int(with_norm)))

    def norm_sum(self) -> float:
        v = C.c_double()
        _check(self.L.piafs_gpu_slab_norm_sum(self.h, C.byref(v)))
        return v.value

    def synchronize(self):
        _check(self.L.piafs_gpu_synchronize(self.sim))

    def solution(self) -> np.ndarray:
        i = self.info
        u = np.empty((i.dim[0] * i.slab_rows, i.nvars))
        _check(self.L.piafs_gpu_get_solution(self.sim, _hp(u)))
        return u

    def cfl(self) -> float:
        c = C.c_double()
        _check(self.L.piafs_gpu_ComputeCFL(self.sim, C.byref(c)))
        return c.value


def run_step(slabs: List[_Slab], exchange, with_norm: bool, sync=lambda: None):
    """One time step of the slabs in `slabs` (all of a grid's slabs, or this
    process's one), `exchange(kind, sends, recvs, send_sizes, recv_sizes)`
    moving the data of each exchange point; `sync` orders the library's
    stream against the torch copies where they run on different streams."""
    lay = slabs[0].layout
    for st in range(slabs[0].info.nstages):
        for s in slabs:
            s.stage_begin(st)
        sync()
        sends, recvs, ss, rs = [], [], [], []
        for s in slabs:
            snd, sz = lay.halo_send(s.rank, s.U[st])
            rsz = lay.halo_recv_sizes(s.rank)
            sends.append(snd)
            ss.append(sz)
            rs.append(rsz)
            recvs.append(snd.new_empty(sum(rsz)))
        exchange("halo", sends, recvs, ss, rs)
        for s, rcv in zip(slabs, recvs):
            lay.halo_apply(s.rank, s.U[st], rcv)
        sends = [lay.column_send(s.U[st]) for s in slabs]
        recvs = [torch_empty_like(x) for x in sends]
        exchange("columns", [x.view(-1) for x in sends], [x.view(-1) for x in recvs], None, None)
        for s, rcv in zip(slabs, recvs):
            lay.column_apply(rcv, s.utc)
        sync()
        for s in slabs:
            s.y_pass(st)
        sync()
        exchange("hy", [s.hy_send for s in slabs], [s.hy_recv for s in slabs], None, None)
        sync()
        for s in slabs:
            s.stage_end(st)
    for s in slabs:
        s.step_end(with_norm)


def torch_empty_like(x):
    import torch
    return torch.empty_like(x)


def local_exchange(sync=lambda: None):
    """The exchange of slabs held in one process: block (src -> dst) of
    every send buffer copied into block (dst <- src) of the receive buffer;
    equal blocks when no sizes are given."""
    def ex(kind, sends, recvs, ss, rs):
        sync()
        P = len(sends)
        if ss is None:
            ss = [[x.numel() // P] * P for x in sends]
            rs = [[x.numel() // P] * P for x in recvs]
        so = [np.concatenate([[0], np.cumsum(z)]).astype(int) for z in ss]
        ro = [np.concatenate([[0], np.cumsum(z)]).astype(int) for z in rs]
        for src in range(P):
            for dst in range(P):
                n = ss[src][dst]
                if n:
                    recvs[dst][ro[dst][src]: ro[dst][src] + n].copy_(sends[src][so[src][dst]: so[src][dst] + n])
        sync()
    return ex


def dist_exchange(group=None, host_staging=False):
    """The exchange of one slab per rank of a torch.distributed group: one
    all_to_all_single per exchange point, on device buffers (NCCL), or
    through host copies for a backend without device collectives (gloo)."""
    import torch.distributed as dist

    def ex(kind, sends, recvs, ss, rs):
        osz, isz = (rs[0] if rs else None), (ss[0] if ss else None)
        if host_staging:
            r = recvs[0].new_empty(recvs[0].shape, device="cpu")
            dist.all_to_all_single(r, sends[0].cpu(), output_split_sizes=osz, input_split_sizes=isz, group=group)
            recvs[0].copy_(r)
        else:
            dist.all_to_all_single(recvs[0], sends[0], output_split_sizes=osz, input_split_sizes=isz, group=group)
    return ex


class LocalSlabs:
    """Every row slab of a grid in this process, on the current device; the
    exchanges are device copies between the slabs' buffers."""

    def __init__(self, deck_dir: str, nranks: int, precision: str = "fp64"):
        self.slabs = [_Slab(deck_dir, precision, r, nranks) for r in range(nranks)]
        self.nranks = nranks

    def close(self):
        for s in self.slabs:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def step(self, nsteps: int = 1):
        import torch
        for _ in range(nsteps):
            run_step(self.slabs, local_exchange(torch.cuda.synchronize), False, torch.cuda.synchronize)
        for s in self.slabs:
            s.synchronize()

    def solution(self) -> np.ndarray:
        """The whole grid's interior solution, (N0 N1, nvars), output order."""
        return np.concatenate([s.solution() for s in self.slabs], axis=0)


class SlabSimulation:
    """This process's row slab of a grid decomposed over the ranks of a
    torch.distributed group (NCCL, one GPU per rank).  Library calls,
    torch copies and collectives all run on the slab's stream."""

    def __init__(self, deck_dir: str, precision: str = "fp64", group=None):
        import torch.distributed as dist
        self.dist, self.group = dist, group
        # a backend without device collectives exchanges through host copies
        self.host_staging = dist.get_backend(group) != "nccl"
        rank, world = dist.get_rank(group), dist.get_world_size(group)
        self.slab = _Slab(deck_dir, precision, rank, world)

    def close(self):
        self.slab.close()

    def step(self, nsteps: int = 1, norm: bool = False) -> Optional[float]:
        """Advance nsteps steps; with norm, the residual norm of the last one
        over the whole grid (TimePostStep.c:36-54)."""
        import torch
        stream = torch.cuda.ExternalStream(self.slab.stream)
        with torch.cuda.stream(stream):
            for k in range(nsteps):
                run_step([self.slab], dist_exchange(self.group, self.host_staging), norm and k == nsteps - 1)
        self.slab.synchronize()
        if not norm:
            return None
        t = torch.tensor([self.slab.norm_sum()], dtype=torch.float64, device=self._coll_device())
        self.dist.all_reduce(t, group=self.group)
        i = self.slab.info
        return float(np.sqrt(t.item() / (i.dim[0] * i.dim[1])))

    def _coll_device(self):
        return "cpu" if self.host_staging else "cuda"

    def state(self) -> np.ndarray:
        """This slab's ghosted state (reference layout, host copy)."""
        i = self.slab.info
        u = np.empty((i.dim[0] + 2 * i.ghosts) * (i.slab_rows + 2 * i.ghosts) * i.nvars)
        _check(self.slab.L.piafs_gpu_get_state(self.slab.sim, _hp(u)))
        return u

    def set_state(self, u: np.ndarray, t: float):
        u = np.ascontiguousarray(u, dtype=np.float64)
        _check(self.slab.L.piafs_gpu_set_state(self.slab.sim, _hp(u), float(t)))

    @property
    def stream(self) -> int:
        return self.slab.stream

    def cfl(self) -> float:
        import torch
        t = torch.tensor([self.slab.cfl()], dtype=torch.float64, device=self._coll_device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)
        return t.item()

    def solution(self) -> np.ndarray:
        """This slab's interior solution (rows of the slab, output order)."""
        return self.slab.solution()

    def gather_solution(self) -> Optional[np.ndarray]:
        """The whole grid's solution on rank 0 (None elsewhere)."""
        parts = [None] * self.dist.get_world_size(self.group)
        self.dist.all_gather_object(parts, self.slab.solution(), group=self.group)
        return np.concatenate(parts, axis=0) if self.dist.get_rank(self.group) == 0 else None
