"""Work split for runs over several GPUs (piafs_b200.shard), on the CPU.

Ensemble members and serving requests are independent units; a rank takes
its share, advances it with no data exchanged, and the per-rank results are
gathered at the end.  These tests check the split (every unit exactly once,
balanced work, the same on every rank) and the gather across two gloo ranks.
"""
import filecmp
import os
import socket

import pytest

from piafs_b200 import cases, shard


def test_balance_covers_every_unit_once_and_balances_work():
    params = cases.ensemble_params(256, steps=100)
    work = [m["side"] ** 2 * m["steps"] for m in params]
    for n in (1, 2, 3, 4, 8):
        parts = shard.balance(work, n)
        assert sorted(i for p in parts for i in p) == list(range(len(work)))
        loads = [sum(work[i] for i in p) for p in parts]
        # longest-processing-time-first: within the largest unit of the mean
        assert max(loads) - sum(loads) / n <= max(work)
        assert shard.balance(work, n) == parts          # deterministic


def test_balance_more_ranks_than_units_and_round_robin():
    parts = shard.balance([3.0, 1.0], 4)
    assert sorted(i for p in parts for i in p) == [0, 1] and sum(1 for p in parts if not p) == 2
    rr = [shard.round_robin(10, r, 3) for r in range(3)]
    assert sorted(i for p in rr for i in p) == list(range(10)) and rr[1] == [1, 4, 7]
    with pytest.raises(ValueError):
        shard.balance([1.0], 0)


def test_ensemble_subset_decks_equal_the_full_ensemble(tmp_path):
    full = cases.ensemble(str(tmp_path / "full"), n=5, steps=3, side_range=(32, 64))
    sub = cases.ensemble(str(tmp_path / "sub"), n=5, steps=3, side_range=(32, 64), members=[1, 4])
    assert [m["index"] for m in sub] == [1, 4]
    for m in sub:
        f = full[m["index"]]
        assert (m["side"], m["dt"], m["Re"]) == (f["side"], f["dt"], f["Re"])
        for name in os.listdir(f["dir"]):
            assert filecmp.cmp(os.path.join(f["dir"], name), os.path.join(m["dir"], name), shallow=False), name


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        params = cases.ensemble_params(64, steps=10)
        mine = shard.balance([m["side"] ** 2 for m in params], world)[rank]
        got = shard.gather({"rank": rank, "members": mine})
        if rank == 0:
            with open(out, "w") as f:
                f.write(repr(got))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_and_gather(tmp_path):
    mp = pytest.importorskip("torch.multiprocessing")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = str(tmp_path / "gathered.txt")
    mp.start_processes(_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    got = eval(open(out).read())
    assert [g["rank"] for g in got] == [0, 1]
    members = [i for g in got for i in g["members"]]
    assert sorted(members) == list(range(64)) and len(set(members)) == 64
    assert got[0]["members"] == shard.balance([m["side"] ** 2 for m in cases.ensemble_params(64, 10)], 2)[0]
