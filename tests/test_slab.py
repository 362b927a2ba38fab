"""The decomposition of a 2D grid into row slabs (piafs_b200/slab.py), on
the CPU: the step driver, the index arithmetic of the three exchanges and
the exchanges themselves, in one process and over two gloo ranks.

Each slab here is a stand-in with the library slab's interface whose
"physics" is chosen so that any misplaced value shows: the y pass sums every
column prefix of its column slab (it needs every row of the grid, ghost rows
included, in order), the stage end adds that sum to the row slab's x-term
(a function of the slab's own rows and the ghost rows the halo exchange
filled).  The result is compared with the same functions evaluated on the
whole grid.  The library's slab runs the same driver on the GPU
(tests/test_gpu_slab.py).
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from piafs_b200.slab import SlabLayout, dist_exchange, local_exchange, run_step


class _Info:
    def __init__(self, nstages):
        self.nstages = nstages


class FakeSlab:
    """Row slab `rank` of the ghosted whole-grid array G[nvars, N1+2g, N0+2g]."""

    def __init__(self, G, rank, nranks, g, periodic, nstages=2):
        nv, W1, W0 = G.shape
        N0, N1 = W0 - 2 * g, W1 - 2 * g
        n1, n0 = N1 // nranks, N0 // nranks
        ps = (n1 + 2 * g) * W0 + 5           # padded planes, as the library's
        psc = (n0 + 2 * g) * W1 + 3
        self.layout = SlabLayout(N0, N1, g, nv, nranks, ps, psc, periodic)
        self.rank, self.g, self.n1, self.n0, self.N0, self.N1 = rank, g, n1, n0, N0, N1
        self.info = _Info(nstages)
        self.G = G
        U = torch.full((nv * ps,), float("nan"), dtype=torch.float64)
        V = self.layout.rows(U)
        V[:, g: g + n1, :] = G[:, g + rank * n1: g + (rank + 1) * n1, :]
        # physical ghost rows (the boundary zones' work) on the end slabs
        if not periodic and rank == 0:
            V[:, 0:g, :] = G[:, 0:g, :]
        if not periodic and rank == nranks - 1:
            V[:, g + n1:, :] = G[:, g + N1:, :]
        self.U = [U] * nstages
        self.utc = torch.full((nv * psc,), float("nan"), dtype=torch.float64)
        self.hy_send = torch.empty(nv * N1 * n0, dtype=torch.float64)
        self.hy_recv = torch.empty(nv * N1 * n0, dtype=torch.float64)
        self.out = []

    def stage_begin(self, st):
        pass

    def y_pass(self, st):
        lay, g = self.layout, self.g
        Cv = lay.cols(self.utc)[:, g: g + self.n0, :]            # [nv, n0, N1 + 2g]
        pre = torch.cumsum(Cv, dim=2)[:, :, g: g + self.N1]      # [nv, n0, N1]
        hy = self.hy_send.view(lay.P, lay.nvars, self.n1, self.n0)
        hy.copy_(pre.reshape(lay.nvars, self.n0, lay.P, self.n1).permute(2, 0, 3, 1))

    def stage_end(self, st):
        lay, g = self.layout, self.g
        V = lay.rows(self.U[st])
        hx = V[:, 2 * g:, g:g + self.N0] - V[:, : -2 * g, g:g + self.N0]   # rows j+g vs j-g: needs the halo
        hy = self.hy_recv.view(lay.P, lay.nvars, self.n1, self.n0).permute(1, 2, 0, 3).reshape(
            lay.nvars, self.n1, self.N0)
        self.out.append((hx + hy).clone())

    def step_end(self, with_norm):
        pass


def expected(G, g):
    N1, N0 = G.shape[1] - 2 * g, G.shape[2] - 2 * g
    hx = G[:, 2 * g:, g:g + N0] - G[:, : -2 * g, g:g + N0]
    hy = torch.cumsum(G[:, :, g:g + N0], dim=1)[:, g:g + N1, :]
    return hx + hy


def whole_grid(nv, N1, N0, g, periodic, seed):
    gen = torch.Generator().manual_seed(seed)
    G = torch.rand((nv, N1 + 2 * g, N0 + 2 * g), generator=gen, dtype=torch.float64)
    if periodic:
        G[:, :g, :] = G[:, N1:N1 + g, :]
        G[:, N1 + g:, :] = G[:, g:2 * g, :]
    return G


@pytest.mark.parametrize("nranks,periodic", [(2, False), (2, True), (3, False), (4, True)])
def test_slabs_in_one_process(nranks, periodic):
    g, nv, N0, N1 = 3, 5, 12 * nranks, 4 * nranks
    G = whole_grid(nv, N1, N0, g, periodic, 7 + nranks)
    slabs = [FakeSlab(G, r, nranks, g, periodic) for r in range(nranks)]
    run_step(slabs, local_exchange(), False)
    got = torch.cat([s.out[-1] for s in slabs], dim=1)
    assert len(slabs[0].out) == 2
    assert torch.equal(got, expected(G, g))


def test_layout_rejects_uneven_grids():
    with pytest.raises(ValueError):
        SlabLayout(10, 9, 3, 4, 2, 100, 100, False)


def _gloo_rank(rank, world, port, periodic, q):
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g, nv, N0, N1 = 3, 4, 8 * world, 5 * world
        G = whole_grid(nv, N1, N0, g, periodic, 11)
        s = FakeSlab(G, rank, world, g, periodic, nstages=3)
        run_step([s], dist_exchange(), False)
        parts = [None] * world
        dist.all_gather_object(parts, s.out[-1])
        if rank == 0:
            q.put(bool(torch.equal(torch.cat(parts, dim=1), expected(G, g))) and len(s.out) == 3)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


@pytest.mark.parametrize("periodic", [False, True])
def test_slabs_over_two_gloo_ranks(periodic):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gloo_rank, args=(r, 2, port, periodic, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=5) is True
