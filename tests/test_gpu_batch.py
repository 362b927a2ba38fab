"""Batched simulations (piafs_gpu_batch_*) against the same decks run alone.

A batch advances many members, of different sizes, physics and step counts,
with one persistent kernel per Runge-Kutta stage.  Its kernels evaluate the
expressions of the single-simulation path, but the compiler contracts
multiply-adds differently in the fused kernel, so a member agrees with its
deck run alone through piafs_gpu_TimeRK to rounding: the FP64 parity bar
(relative L2 <= 1e-12 per variable, variables without signal held to it in
absolute terms).  A tile's arithmetic depends only on its own member, so a
member's result is bit for bit the same alone in a batch, in any mix, and
whenever it joins.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from piafs_b200 import Batch, PiafsError, Simulation, cases, deck

pytestmark = pytest.mark.gpu

GOLDEN_WENO = ["euler1d_weno5_roe_n1024", "euler1d_weno5_llf_yc_rk4_n128", "ns2d_chem_weno5_llf_48x40",
               "ns2d_shear_weno5_roe_re200_40x32"]


TOL = 1e-12
NOISE_FLOOR = 1e-6
MIXED_TOL = 1e-5
# tile shapes of the stage kernel (x, y)
SHAPES = [(16, 16), (32, 8), (16, 8), (32, 4), (8, 16), (16, 15), (32, 7), (16, 7)]


def rel_err(got, ref):
    """Worst relative L2 over the variables (variables without signal in
    absolute terms against the largest variable's RMS)."""
    rms = np.sqrt((ref * ref).mean(axis=0))
    scale = rms.max()
    worst = 0.0
    for v in range(ref.shape[1]):
        d = got[:, v] - ref[:, v]
        if rms[v] < NOISE_FLOOR * scale:
            err = np.sqrt((d * d).mean()) / scale
        else:
            err = np.sqrt((d * d).sum() / (ref[:, v] ** 2).sum())
        worst = max(worst, err)
    return worst


def assert_close(got, ref, what=""):
    rms = np.sqrt((ref * ref).mean(axis=0))
    scale = rms.max()
    worst = 0.0
    for v in range(ref.shape[1]):
        d = got[:, v] - ref[:, v]
        if rms[v] < NOISE_FLOOR * scale:
            err = np.sqrt((d * d).mean()) / scale
        else:
            err = np.sqrt((d * d).sum() / (ref[:, v] ** 2).sum())
        worst = max(worst, err)
    assert np.all(np.isfinite(got)) and worst <= TOL, f"{what}: {worst:.2e}"


def in_batch_alone(d, steps, tile_x=0, precision="fp64"):
    with Batch(precision) as b:
        if tile_x:
            b.tune(tile_x)
        i = b.add(d, steps)
        b.step(steps)
        return b.solution(i)


def alone(d, steps):
    with Simulation(d) as s:
        s.time_rk(steps)
        return s.solution()


def make_mix(root):
    """Small decks of every member kind, sizes off the tile grid."""
    out = []
    for k, (n, ny, amp) in enumerate([(96, 96, 0.7), (64, 160, 1.3), (50, 37, 1.0)]):
        d = os.path.join(root, f"beam{k}")
        cases.ns2d_photochem_beam(d, N=n, NY=ny, n_iter=12, scheme="weno5", op_file_format="none",
                                  dt=0.4 / 2048, beam_amp=amp, seed=k)
        out.append((d, 12))
    d = os.path.join(root, "euler300")
    cases.euler1d_density_wave(d, N=300, n_iter=40, dt=1e-4, scheme="weno5", op_file_format="none")
    out.append((d, 40))
    for name in GOLDEN_WENO:
        d = os.path.join(GOLDEN, name)
        n = int(deck.read_keyfile(os.path.join(d, "solver.inp"))["n_iter"][0])
        out.append((d, min(n, 60)))
    return out


def test_batch_members_match_single_runs(tmp_path):
    mix = make_mix(str(tmp_path))
    with Batch() as b:
        ids = [b.add(d, n) for d, n in mix]
        assert b.info["members"] == len(mix)
        b.step(max(n for _, n in mix))
        done = b.poll()
        assert sorted(done) == sorted(ids)
        for (d, n), i in zip(mix, ids):
            m = b.member(i)
            assert m["iter"] == n and m["done"]
            got = b.solution(i)
            assert_close(got, alone(d, n), d)
            # the mix does not change a member's bits
            assert np.array_equal(got, in_batch_alone(d, n)), d


def test_batch_golden_decks_match_the_reference():
    """Full-length golden WENO5 runs in one batch against the reference's
    own output (the FP64 parity bar)."""
    with Batch() as b:
        ids = {name: b.add(os.path.join(GOLDEN, name)) for name in GOLDEN_WENO}
        b.step(1000)
        for name, i in ids.items():
            got = b.solution(i)
            ref = deck.read_op(os.path.join(GOLDEN, name, "ref_final.bin")).u
            num = np.sqrt(((got - ref) ** 2).sum(axis=0))
            den = np.sqrt((ref ** 2).sum(axis=0))
            rel = np.where(den > 1e-15, num / np.maximum(den, 1e-300), num)
            assert rel.max() <= 1e-12, (name, rel)


def test_continuous_batching_join_leave(tmp_path):
    """Members join while others run and leave when done; each result is bit
    for bit the result of the member alone in a batch."""
    mix = make_mix(str(tmp_path))
    with Batch() as b:
        first = [b.add(d, n) for d, n in mix[:3]]
        b.step(5)
        later = [b.add(d, n) for d, n in mix[3:]]
        finished = []
        for _ in range(200):
            b.step(3)
            finished += b.poll()
            if len(finished) == len(mix):
                break
        assert sorted(finished) == sorted(first + later)
        for (d, n), i in zip(mix, first + later):
            assert np.array_equal(b.solution(i), in_batch_alone(d, n)), d
        for i in first:
            b.remove(i)
        assert b.info["members"] == len(later)


@pytest.mark.parametrize("tile_x", [16, 32, 8])
def test_tile_shapes(tmp_path, tile_x):
    mix = make_mix(str(tmp_path))[:4]
    with Batch() as b:
        b.tune(tile_x)
        ids = [b.add(d, n) for d, n in mix]
        b.step(max(n for _, n in mix))
        assert b.info["tile_x"] == tile_x
        for (d, n), i in zip(mix, ids):
            got = b.solution(i)
            assert_close(got, alone(d, n), d)
            assert np.array_equal(got, in_batch_alone(d, n, tile_x)), d


def test_budget_admission_and_rejections(tmp_path):
    d = os.path.join(str(tmp_path), "b")
    cases.ns2d_photochem_beam(d, N=64, n_iter=4, scheme="weno5", op_file_format="none", dt=0.4 / 2048)
    with Batch(hbm_budget_bytes=1) as b:
        with pytest.raises(PiafsError) as ex:
            b.add(d)
        assert ex.value.code == 7
    with Batch() as b:
        i = b.add(d)
        one = b.info["bytes_in_use"]
    with Batch(hbm_budget_bytes=int(one * 1.5)) as b:
        i = b.add(d)
        with pytest.raises(PiafsError):
            b.add(d)
        b.step(4)
        assert b.poll() == [i]
        b.remove(i)
        b.add(d)                      # memory freed: admitted again
    c = os.path.join(str(tmp_path), "c")
    cases.ns2d_photochem_beam(c, N=64, n_iter=4, scheme="crweno5", op_file_format="none", dt=0.4 / 2048)
    with Batch() as b:
        with pytest.raises(PiafsError) as ex:
            b.add(c)
        assert ex.value.code == 3


def test_autotuner_restores_state_and_picks_a_config(tmp_path):
    mix = make_mix(str(tmp_path))[:5]
    with Batch() as b:
        ids = b.add_many([d for d, _ in mix], [n for _, n in mix])
        b.step(3)
        before = [b.solution(i) for i in ids]
        iters = [b.member(i)["iter"] for i in ids]
        b.tune()
        assert [b.member(i)["iter"] for i in ids] == iters
        for i, u in zip(ids, before):
            assert np.array_equal(b.solution(i), u)
        info = b.info
        assert (info["tile_x"], info["tile_y"]) in SHAPES and info["min_ctas_per_sm"] in (1, 2)
        b.step(200)
        for (d, n), i in zip(mix, ids):
            assert_close(b.solution(i), alone(d, n), d)
        # the same configuration set explicitly gives the same bits
        with Batch() as c:
            c.set_launch(info["tile_x"], info["tile_y"], info["min_ctas_per_sm"])
            j = c.add(mix[0][0], mix[0][1])
            c.step(mix[0][1])
            assert np.array_equal(c.solution(j), b.solution(ids[0]))


def test_persistent_ctas_walking_many_tiles(tmp_path, monkeypatch):
    """One persistent CTA walks every tile of members whose sides are not
    multiples of the tile (partial edge tiles), through all RK stages: the
    results are those of the full grid of CTAs, bit for bit, and of the
    single-simulation path to the parity bar."""
    decks = []
    for k, (n, ts) in enumerate([(117, "ssprk3"), (100, "22"), (75, "44")]):
        d = os.path.join(str(tmp_path), f"p{k}")
        cases.ns2d_photochem_beam(d, N=n, n_iter=3, scheme="weno5", dt=8e-5, time_scheme_type=ts,
                                  op_file_format="none", seed=k)
        decks.append(d)
    e = os.path.join(str(tmp_path), "e")
    cases.euler1d_density_wave(e, N=1500, n_iter=3, dt=1e-4, scheme="weno5", op_file_format="none")
    decks.append(e)

    def run():
        with Batch() as b:
            ids = [b.add(d, 3) for d in decks]
            b.step(3)
            return [b.solution(i) for i in ids]

    full = run()
    monkeypatch.setenv("PIAFS_GPU_BATCH_GRID", "1")
    one = run()
    for d, a, b in zip(decks, full, one):
        assert np.array_equal(a, b), d
        assert_close(a, alone(d, 3), d)


def test_mixed_precision_members_track_fp64(tmp_path):
    """Mixed-precision members (FP32 weights, reconstruction, upwind fluxes,
    viscous stencils and chemistry on FP64 state and RK accumulation) stay
    within MIXED_TOL relative L2 of the FP64 single runs, and a member's
    result is bit for bit the same alone and in the mix."""
    mix = make_mix(str(tmp_path))
    with Batch("mixed") as b:
        ids = [b.add(d, n) for d, n in mix]
        b.step(max(n for _, n in mix))
        assert sorted(b.poll()) == sorted(ids)
        for (d, n), i in zip(mix, ids):
            got = b.solution(i)
            assert np.all(np.isfinite(got)), d
            err = rel_err(got, alone(d, n))
            print(f"{os.path.basename(d)}: mixed batch vs FP64 rel L2 {err:.2e}")
            assert err <= MIXED_TOL, (d, err)
            assert np.array_equal(got, in_batch_alone(d, n, precision="mixed")), d


@pytest.mark.parametrize("tile", [(16, 15, 1), (16, 7, 2), (32, 7, 1)])
def test_balanced_tiles_both_precisions(tmp_path, tile):
    """The 15- and 7-row tiles (at most one interface per thread) in FP64 and
    mixed precision, on members whose sides are not multiples of the tile."""
    mix = make_mix(str(tmp_path))[:4]
    for prec in ("fp64", "mixed"):
        with Batch(prec) as b:
            b.set_launch(*tile)
            ids = [b.add(d, n) for d, n in mix]
            b.step(max(n for _, n in mix))
            assert (b.info["tile_x"], b.info["tile_y"]) == tile[:2]
            for (d, n), i in zip(mix, ids):
                got = b.solution(i)
                if prec == "fp64":
                    assert_close(got, alone(d, n), d)
                else:
                    assert rel_err(got, alone(d, n)) <= MIXED_TOL, d


def test_mixed_persistent_ctas_walking_many_tiles(tmp_path, monkeypatch):
    """Mixed precision with one persistent CTA walking all tiles gives the
    bits of the full grid of CTAs."""
    decks = []
    for k, n in enumerate([117, 75]):
        d = os.path.join(str(tmp_path), f"p{k}")
        cases.ns2d_photochem_beam(d, N=n, n_iter=3, scheme="weno5", dt=8e-5, op_file_format="none", seed=k)
        decks.append(d)

    def run():
        with Batch("mixed") as b:
            ids = [b.add(d, 3) for d in decks]
            b.step(3)
            return [b.solution(i) for i in ids]

    full = run()
    monkeypatch.setenv("PIAFS_GPU_BATCH_GRID", "1")
    one = run()
    for d, a, c in zip(decks, full, one):
        assert np.array_equal(a, c), d
