"""Request serving: parameter-described solves, continuous batching, budget.

A request's deck is written in memory and its fields generated on the
device; it must reproduce the same solve set up from the case generator's
deck files (the fields agree up to the last bit of sin / exp), and it must
give the same result, bit for bit, alone and in the served mix (checksums
through the serving loop, whole solutions through the same continuous
batching driven step by step; FP64 and mixed precision).
"""
import os

import numpy as np
import pytest

from piafs_b200 import (REQUEST_EULER1D_WAVE, REQUEST_NS2D_BEAM, Batch, PiafsError, Request, Simulation, cases,
                        serve_trace)

pytestmark = pytest.mark.gpu


def rel_l2(got, ref):
    num = np.sqrt(((got - ref) ** 2).sum(axis=0))
    den = np.sqrt((ref ** 2).sum(axis=0))
    return np.where(den > 1e-15, num / np.maximum(den, 1e-300), num).max()


def one(req, precision="fp64"):
    with Batch(precision=precision) as b:
        i = b.add_request(req)
        b.step(req.nsteps)
        return b.solution(i), b.checksum(i)


def test_requests_reproduce_deck_runs(tmp_path):
    d1 = str(tmp_path / "e")
    cases.euler1d_density_wave(d1, N=200, n_iter=30, dt=0.1 / 200, amp=0.2, op_file_format="none")
    got, _ = one(Request(kind=REQUEST_EULER1D_WAVE, n=200, nsteps=30, dt=0.1 / 200, amp=0.2))
    with Simulation(d1) as s:
        s.time_rk(30)
        assert rel_l2(got, s.solution()) <= 1e-12
    d2 = str(tmp_path / "b")
    Re, side = 3.0e4, 48
    theta = np.arcsin(np.sin(cases.THETA_RE_1E4) * 1e4 / Re)
    dt = min(0.4 / side, (0.4 / 2048) * 1e4 / Re)
    cases.ns2d_photochem_beam(d2, N=side, n_iter=25, scheme="weno5", beam_amp=1.1, beam_radius=0.07, theta=theta,
                              Re=Re, dt=dt, noise=0.0, op_file_format="none")
    got, _ = one(Request(kind=REQUEST_NS2D_BEAM, n=side, nsteps=25, dt=dt, amp=1.1, beam_radius=0.07, Re=Re,
                         noise=0.0, seed=5))
    with Simulation(d2) as s:
        s.time_rk(25)
        ref = s.solution()
    rms = np.sqrt((ref * ref).mean(axis=0))
    sig = rms >= 1e-6 * rms.max()
    num = np.sqrt(((got - ref) ** 2).sum(axis=0))
    den = np.sqrt((ref ** 2).sum(axis=0))
    assert (num[sig] / den[sig]).max() <= 1e-12
    assert (np.sqrt(((got - ref) ** 2).mean(axis=0))[~sig] / rms.max()).max(initial=0.0) <= 1e-12


def small_trace(n=40):
    reqs, arr = cases.serving_trace(n=n, rate=400.0, n1d=(64, 512), side2d=(32, 96), steps=(10, 40))
    return [Request(**r) for r in reqs], arr


def test_served_results_equal_alone_results():
    reqs, arr = small_trace()
    res = serve_trace(reqs, arr, steps_per_round=3)
    assert all(r["finished_s"] >= r["admitted_s"] >= 0 for r in res)
    assert all(r["admitted_s"] >= r["arrival_s"] - 1e-6 for r in res)
    for q, r in zip(reqs, res):
        assert r["steps"] == q.nsteps
        _, cs = one(q)
        assert r["checksum"] == cs


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_served_checksums_equal_alone_checksums(precision):
    reqs, arr = small_trace(24)
    res = serve_trace(reqs, arr, precision=precision, steps_per_round=3)
    for q, r in zip(reqs, res):
        _, cs = one(q, precision)
        assert r["checksum"] == cs


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_continuous_batching_full_solutions_equal_alone(precision):
    """The serving loop's pattern -- requests joining a batch whose other
    members are part-way through their steps, finished members polled out
    and removed while the rest go on -- leaves every member's whole solution
    bit for bit as it is alone."""
    reqs, _ = small_trace(16)
    alone = [one(q, precision)[0] for q in reqs]
    got = {}
    with Batch(precision=precision) as b:
        ids = {}
        pending = list(range(len(reqs)))
        while pending or ids:
            for _ in range(min(3, len(pending))):       # a few arrivals per round
                k = pending.pop(0)
                ids[b.add_request(reqs[k])] = k
            b.step(2)
            for i in b.poll():
                got[ids[i]] = b.solution(i)
                b.remove(i)
                del ids[i]
    assert sorted(got) == list(range(len(reqs)))
    for k, ref in enumerate(alone):
        assert np.array_equal(got[k], ref), (k, precision)


def test_serving_under_a_small_budget():
    """With room for only a few requests at a time, requests wait for memory
    and every one still completes with the result it has alone."""
    reqs, arr = small_trace(24)
    sizes = []
    with Batch() as b:
        for q in reqs:
            i = b.add_request(q)
            sizes.append(b.info["bytes_in_use"])
            b.remove(i)
    res = serve_trace(reqs, arr, hbm_budget_bytes=3 * max(sizes), steps_per_round=2)
    for q, r in zip(reqs, res):
        _, cs = one(q)
        assert r["checksum"] == cs
    # a request larger than the whole budget is refused, not waited on forever
    with pytest.raises(PiafsError):
        serve_trace(reqs[:1], arr[:1], hbm_budget_bytes=16)


def test_resident_points_bound():
    """With the resident grid points bounded, requests are admitted in arrival
    order as earlier ones finish (never more points resident than the bound,
    except one request alone), and each result is still its result alone."""
    reqs, arr = small_trace(30)
    pts = [q.n if q.kind == 1 else q.n * q.n for q in reqs]
    bound = 2 * max(pts)
    res = serve_trace(reqs, arr, steps_per_round=2, max_resident_points=bound)
    adm = [r["admitted_s"] for r in res]
    assert adm == sorted(adm)
    for k, r in enumerate(res):
        # requests resident at k's admission: admitted no later, finished after
        live = [j for j in range(len(res)) if res[j]["admitted_s"] <= r["admitted_s"] < res[j]["finished_s"]]
        assert sum(pts[j] for j in live) <= max(bound, pts[k])
    for q, r in zip(reqs, res):
        _, cs = one(q)
        assert r["checksum"] == cs
