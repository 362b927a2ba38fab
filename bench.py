#!/usr/bin/env python
"""Benchmark of the PIAFS per-stage RHS + explicit RK path on B200.

Metric: grid-point RK-stage updates per second (one unit = one interior grid
point advanced through one Runge-Kutta stage).  Default workload: the 2D
Navier-Stokes photochemical case on a 2048 x 2048 grid (11 conserved
variables, CRWENO5 components, LLF upwinding, SSPRK3, FP64), synthetic seeded
inputs of that shape.  A "step" is one SSPRK3 time step over the whole grid.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gpu|reference]

With N > 1 (torchrun, one process per GPU) every rank advances its own
independent replica of the workload (replicas are the weakly scaled unit)
and the timed region is bracketed by barriers with the max over ranks taken
on the device clocks.  --workload slab instead decomposes the one grid over
the N ranks (row slabs with NCCL exchanges, strong scaling).

--impl reference times the reference's own CPU implementation (the
llnl/piafs binary built from source by oracle/Makefile, OpenMP on all host
threads) on a bounded sample of the same workload; under torchrun only rank 0
runs it.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_PER_UNIT = {11: 264, 4: 96, 3: 72}   # 3 * nvars * 8: read U_s, read u_n, write (FP64 state)
# measured DRAM traffic of one CRWENO5 line-solve launch per interior point
# (dram__bytes_read + dram__bytes_write, ncu at 1536^2, 11 variables, the
# passive variables' interface values packed)
TRAFFIC_PER_POINT = {11: (416.9e6 + 523.2e6) / (1536 * 1536)}
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
CPU_SAMPLE_N = 512                          # sample grid of the CPU arms
# Steps timed back to back from the initial condition before the state is
# reset to it.  At dt = 0.4 dx the CRWENO5/LLF/SSPRK3 case (CFL 0.4 per
# direction, 0.8 summed over the two) lies beyond the scheme's linear
# stability limit at these resolutions: seeded noise grows into NaN after
# about 24 steps at 2048^2 (in the reference's algorithm and in this one
# alike) and after 9 at 4096^2, where the growth sets in from step 4.  Timing
# chunks from the initial state keep every timed step a finite step of the
# workload (and the mixed-precision error a comparison of smooth states).
def chunk_steps(n):
    return 12 if n <= 2048 else 4 if n <= 4096 else 2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--workload", default="ns2d_photochem",
                    choices=["ns2d_photochem", "euler1d", "ensemble", "serving", "slab"])
    ap.add_argument("--requests", type=int, default=1000, help="serving requests (the stream's first n)")
    ap.add_argument("--hbm-budget-gb", type=float, default=120.0)
    ap.add_argument("--max-resident-points", type=float, default=4e6,
                    help="serving: grid points resident at once (0: HBM budget only)")
    ap.add_argument("--members", type=int, default=256, help="ensemble members")
    ap.add_argument("--member-steps", type=int, default=100, help="steps per ensemble member")
    ap.add_argument("--launch", default=None,
                    help="ensemble: launch configuration TXxTYxCTAS (tile, CTAs per SM) instead of the autotuner's")
    ap.add_argument("--n", type=int, default=None, help="grid size (default 2048 / 1024)")
    ap.add_argument("--scheme", default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-extras", action="store_true",
                    help="leave out the mixed-precision and small-ensemble figures of the default run")
    return ap.parse_args()


def make_deck(path, a, n_iter, n=None):
    from piafs_b200 import cases
    if a.workload == "euler1d":
        N = n or a.n or 1024
        return cases.euler1d_density_wave(path, N=N, n_iter=n_iter, dt=1e-4, scheme=a.scheme or "weno5",
                                          op_file_format="none")
    # CFL 0.4 on this grid (sound speed 1): dt = 0.4 / N
    N = n or a.n or 2048
    return cases.ns2d_photochem_beam(path, N=N, n_iter=n_iter, scheme=a.scheme or "crweno5",
                                     op_file_format="none", dt=0.4 / N)


def workload_config(a, meta, n_gpus):
    sz = meta["size"]
    name = ("ns2d_photochem_crweno5_llf_ssprk3" if a.workload == "ns2d_photochem" else "euler1d_weno5_roe_ssprk3")
    if a.scheme:
        name = name.replace("crweno5", a.scheme).replace("weno5", a.scheme)
    return {"workload": f"{name}_{'x'.join(map(str, sz))}", "grid": sz, "nvars": meta["nvars"],
            "time_scheme": "ssprk3", "dt": meta["dt"], "replicas": n_gpus, "parallelism": f"replicas{n_gpus}",
            "precision": a.precision,
            "step": "one SSPRK3 time step (3 RK stages) over the whole grid",
            "timing": f"chunks of at most {chunk_steps(sz[0])} steps from the initial condition, device time summed",
            "l2": "state arrays (%.0f MB each) exceed the 126 MB L2; no flush" % (
                8 * meta["nvars"] * (sz[0] + 6) * ((sz[1] + 6) if len(sz) > 1 else 1) / 1e6)}


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.idx), "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------ CPU baselines
def ref_binary():
    for b in ("PIAFS_omp", "PIAFS"):
        p = os.path.join(REF_DIR, b)
        if os.access(p, os.X_OK):
            return p, b == "PIAFS_omp"
    return None, False


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def sample_size(nsteps, warm):
    """Grid side of the CPU sample: the whole reference run should take about
    two minutes at ~0.2 M updates/s (the reference's rate on this workload)."""
    budget = 120.0 / max(nsteps + warm, 1)
    n = int((budget * 0.2e6 / 3) ** 0.5) // 32 * 32
    return max(128, min(CPU_SAMPLE_N, n))


def run_reference_steps(a, nsteps, warm):
    """Run the reference binary on the CPU sample deck; returns (per-step
    seconds of the timed steps, cores, kind, sample description)."""
    binary, omp = ref_binary()
    cores = host_threads() if omp else 1
    with tempfile.TemporaryDirectory() as d:
        n = sample_size(nsteps, warm) if a.workload == "ns2d_photochem" else (a.n or 1024)
        meta = make_deck(d, a, warm + nsteps, n=n)
        # per-step wall time lines: "iter= ... wctime: X (s)" (TimePrintStep.c)
        from piafs_b200 import deck
        kv = deck.read_keyfile(os.path.join(d, "solver.inp"))
        txt = open(os.path.join(d, "solver.inp")).read()
        txt = re.sub(r"screen_op_iter\s+\d+", "screen_op_iter 1", txt)
        open(os.path.join(d, "solver.inp"), "w").write(txt)
        if binary:
            env = dict(os.environ, OMP_NUM_THREADS=str(cores))
            out = subprocess.run([binary], cwd=d, env=env, capture_output=True, text=True, check=True).stdout
            w = [float(x) for x in re.findall(r"wctime:\s*([0-9.Ee+-]+)", out)]
            kind = "reference"
        else:
            # the reference binary was not built here: time the oracle port
            from oracle import oracle
            case = oracle.load(d)
            w = []
            u = case.u0.copy()
            for k in range(warm + nsteps):
                t0 = time.perf_counter()
                u = case.run(nsteps=1, u=u, t0=k * case.dt)
                w.append(time.perf_counter() - t0)
            kind, cores = "port", 1
        units = 3 * meta["size"][0] * (meta["size"][1] if len(meta["size"]) > 1 else 1)
        sample = (f"{'x'.join(map(str, meta['size']))} grid of the same workload, {nsteps} timed SSPRK3 steps "
                  f"after {warm} warm-up, per-step wall time printed by the reference")
        return w[warm:warm + nsteps], units, cores, kind, sample


def cpu_baseline(a):
    steps = 3 if a.workload == "ns2d_photochem" else 200
    w, units, cores, kind, sample = run_reference_steps(a, steps, 1)
    v = units * len(w) / sum(w)
    return {"value": v, "unit": "pt-stage updates/s", "cores": cores, "kind": kind, "sample": sample}


# ----------------------------------------------------------------- ensemble
def rel_l2_noise_floor(got, ref, floor=1e-6):
    import numpy as np
    rms = np.sqrt((ref * ref).mean(axis=0))
    scale = rms.max()
    worst = 0.0
    for v in range(ref.shape[1]):
        d = got[:, v] - ref[:, v]
        if rms[v] < floor * scale:
            e = np.sqrt((d * d).mean()) / scale
        else:
            e = np.sqrt((d * d).sum() / (ref[:, v] ** 2).sum())
        worst = max(worst, float(e))
    return worst


def _dist_setup():
    """(rank, world, barrier): one process per GPU under torchrun; the
    process group only brackets the timed regions and gathers results."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
    return rank, world, barrier


def ensemble_bench(a):
    """The batched ensemble: every member of cases.ensemble solved (deck read,
    device set-up, steps, solution back to the host) in one batch, against
    the same members solved one at a time through Simulation (FP64).  Both
    are wall-clock times of complete solves; the batched step phase is also
    reported as grid-point RK-stage updates per second.  Under torchrun the
    members are split across the ranks by work (piafs_b200.shard.balance),
    each rank solves its share, and the times are the max over ranks between
    barriers; only the per-rank results are gathered at the end."""
    import numpy as np
    import torch
    from piafs_b200 import Batch, Simulation, cases, shard

    rank, world, barrier = _dist_setup()
    torch.cuda.init()
    n, steps = a.members, a.member_steps
    params = cases.ensemble_params(n=n, steps=steps)
    mine = shard.balance([m["side"] ** 2 * steps for m in params], world)[rank]
    tmp = tempfile.mkdtemp(prefix=f"piafs_ensemble_r{rank}_")
    try:
        mem = cases.ensemble(tmp, n=n, steps=steps, members=mine)
        sides = [m["side"] for m in mem]
        npts = sum(s * s for s in sides)
        nm = len(mem)
        # warm the CUDA context and the kernels' modules outside the timing
        if nm:
            with Batch(precision=a.precision) as B:
                B.add(mem[0]["dir"], 1)
                B.step(1)
            with Simulation(mem[0]["dir"]) as s:
                s.time_rk(1)
        torch.cuda.synchronize()
        # the launch configuration for this class of ensemble (the autotuner,
        # run once on the full mix; its choice is reused by later ensembles
        # of the class, so it is timed apart from the solves), or the one
        # given with --launch
        t0 = time.perf_counter()
        if a.launch:
            tx, ty, mb = (int(x) for x in a.launch.split("x"))
            tuned = {"tile_x": tx, "tile_y": ty, "min_ctas_per_sm": mb}
        else:
            with Batch(precision=a.precision) as B:
                if nm:
                    B.add_many([m["dir"] for m in mem], [steps] * nm)
                B.tune()
                tuned = B.info
        tune_s = time.perf_counter() - t0
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        with Batch(precision=a.precision) as B:
            B.set_launch(tuned["tile_x"], tuned["tile_y"], tuned["min_ctas_per_sm"])
            ids = B.add_many([m["dir"] for m in mem], [steps] * nm) if nm else []
            t1 = time.perf_counter()
            B.step(steps)
            t2 = time.perf_counter()
            sols = [B.solution(i) for i in ids]
            t3 = time.perf_counter()
            binfo = B.info
        barrier()
        batched = time.perf_counter() - t0
        t0s = time.perf_counter()
        one = []
        for m in mem:
            with Simulation(m["dir"]) as s:
                s.time_rk(steps)
                one.append(s.solution())
        barrier()
        single = time.perf_counter() - t0s
        worst = 0.0
        for sb, so in zip(sols, one):
            worst = max(worst, rel_l2_noise_floor(sb, so))
        finite = all(bool(np.isfinite(x).all()) for x in sols)
        mine_res = {"members": [m["index"] for m in mem], "points": npts, "batched": batched,
                    "single": single, "admit": t1 - t0, "step": t2 - t1, "results": t3 - t2, "worst": worst,
                    "finite": finite, "tune_s": tune_s}
        allr = shard.gather(mine_res)
        if rank != 0:
            return 0
        done = sorted(k for r in allr for k in r["members"])
        assert done == list(range(n)), "every member solved exactly once"
        batched = max(r["batched"] for r in allr)
        single = max(r["single"] for r in allr)
        step_s = max(r["step"] for r in allr)
        total_pts = sum(r["points"] for r in allr)
        all_sides = [m["side"] for m in params]
        units = 3 * steps * total_pts
        line = {"metric": "ensemble solves/s", "value": n / batched, "unit": "solves/s", "n_gpus": world,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "f64" if a.precision == "fp64" else "f32+f64",
                "data": "synthetic (seeded ensemble decks)",
                "config": {"workload": f"ensemble_{n}_ns2d_photochem_weno5_llf_ssprk3_{steps}steps",
                           "members": n, "steps": steps, "sides": [min(all_sides), max(all_sides)],
                           "total_points": total_pts, "precision": a.precision,
                           "tile": [binfo["tile_x"], binfo["tile_y"]],
                           "min_ctas_per_sm": binfo["min_ctas_per_sm"],
                           "tune_s": max(r["tune_s"] for r in allr),
                           "launches_per_step": binfo["launches_per_step"],
                           "parallelism": f"members split by work over {world} GPU(s)",
                           "members_per_rank": [len(r["members"]) for r in allr]},
                "batched": {"wall_s": batched, "admit_s": max(r["admit"] for r in allr),
                            "step_s": step_s, "pt_stage_updates_per_s": units / step_s,
                            "results_s": max(r["results"] for r in allr)},
                "one_at_a_time": {"wall_s": single, "solves_per_s": n / single, "precision": "fp64"},
                "speedup_vs_one_at_a_time": single / batched,
                "accuracy": {"max_rel_l2_vs_one_at_a_time": max(r["worst"] for r in allr)},
                "finite": all(r["finite"] for r in allr)}
        print(json.dumps(line))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return 0


# ------------------------------------------------------------------ serving
def serving_bench(a):
    """The request stream of cases.serving_trace (Poisson arrivals at 2000
    requests/s, 70% 1D Euler / 30% 2D photochemical, 50-500 steps), its first
    --requests requests replayed in real time through the continuous-batching
    serving loop under the HBM budget.  Latency = result ready - arrival.
    Under torchrun request k goes to rank k mod N (each rank serves a Poisson
    stream of rate / N against its own budget); latencies are gathered."""
    import numpy as np
    import torch
    from piafs_b200 import Request, serve_trace, cases, shard

    rank, world, barrier = _dist_setup()
    torch.cuda.init()
    reqs, arr = cases.serving_trace(n=a.requests)
    mine = shard.round_robin(len(reqs), rank, world)
    rq = [Request(**reqs[k]) for k in mine]
    my_arr = [float(arr[k]) for k in mine]
    # warm the context and the kernels
    if rq:
        serve_trace(rq[:2], [0.0] * len(rq[:2]), precision=a.precision)
    budget = int(a.hbm_budget_gb * 1e9)
    maxpts = int(a.max_resident_points)
    barrier()
    t0 = time.perf_counter()
    res = serve_trace(rq, my_arr, precision=a.precision, hbm_budget_bytes=budget, steps_per_round=4,
                      max_resident_points=maxpts) if rq else []
    wall = time.perf_counter() - t0
    barrier()
    allr = shard.gather({"res": res, "wall": wall, "idx": mine})
    if rank != 0:
        return 0
    res = [r for g in allr for r in g["res"]]
    assert sorted(k for g in allr for k in g["idx"]) == list(range(len(reqs))), "every request served once"
    wall = max(g["wall"] for g in allr)
    lat = np.array([r["finished_s"] - r["arrival_s"] for r in res])
    wait = np.array([r["admitted_s"] - r["arrival_s"] for r in res])
    units = sum(3 * q["nsteps"] * (q["n"] if q["kind"] == 1 else q["n"] ** 2) for q in reqs)
    span = max(r["finished_s"] for r in res) - min(r["arrival_s"] for r in res)
    line = {"metric": "served solves/s", "value": len(res) / span, "unit": "solves/s", "n_gpus": world,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64" if a.precision == "fp64" else "f32+f64", "data": "synthetic (seeded request stream)",
            "config": {"workload": f"serving_{len(res)}req_poisson2000_70pct1d_30pct2d_50to500steps",
                       "requests": len(res), "rate_per_s": 2000.0, "precision": a.precision,
                       "hbm_budget_gb": a.hbm_budget_gb, "steps_per_round": 4,
                       "max_resident_points": maxpts, "admission": "FIFO",
                       "parallelism": f"request k on GPU k mod {world}",
                       "pt_stage_updates": units},
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "max": float(lat.max())},
            "queue_wait_s": {"p50": float(np.percentile(wait, 50)), "p99": float(np.percentile(wait, 99))},
            "makespan_s": span, "wall_s": wall, "pt_stage_updates_per_s": units / span,
            "finite": bool(all(np.isfinite(r["checksum"]) for r in res))}
    print(json.dumps(line))
    return 0


# --------------------------------------------------------------------- main
def mixed_figure(tmp, a, fp64_sim, u0, t0, N, fp64_ms_per_step):
    """The same workload in mixed precision (FP32 reconstruction rows,
    weights, fluxes, viscous and source terms on FP64 state, FP64 line
    solves): device time per step over the same chunks as the FP64 timing,
    the ratio over FP64, and the error against the FP64 path after one full
    chunk of steps from the same initial state."""
    import numpy as np
    import torch
    from piafs_b200 import Simulation
    with Simulation(tmp, precision="mixed") as sim:
        stream = torch.cuda.ExternalStream(sim.stream)
        for _ in range(3):
            sim.set_state(u0, t0)
            sim.time_rk(chunk_steps(N))
        ms, done = 0.0, 0
        while done < a.steps:
            n = min(chunk_steps(N), a.steps - done)
            sim.set_state(u0, t0)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sim.time_rk_async(n)
            e1.record(stream)
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            done += n
        k = chunk_steps(N)
        sim.set_state(u0, t0)
        sim.time_rk(k)
        got = sim.solution()
    fp64_sim.set_state(u0, t0)
    fp64_sim.time_rk(k)
    ref = fp64_sim.solution()
    rms = np.sqrt((ref * ref).mean(axis=0))
    sig = rms >= 1e-6 * rms.max()
    l2 = np.sqrt(((got - ref) ** 2).sum(axis=0) / np.maximum((ref * ref).sum(axis=0), 1e-300))
    linf = np.abs(got - ref).max(axis=0) / np.maximum(np.abs(ref).max(axis=0), 1e-300)
    step = ms / a.steps
    return {"ms_per_step": step, "speedup_over_fp64": fp64_ms_per_step / step,
            "error_vs_fp64": {"steps": k, "rel_l2_max": float(l2[sig].max()), "rel_linf_max": float(linf[sig].max())}}


def ensemble_figure(members=32, steps=20):
    """A small instance of the batched ensemble (seeded members of the
    ensemble workload, sides 64-512, WENO5/LLF/SSPRK3, FP64): complete solves
    (deck read, device set-up, steps, solution back) in one batch against the
    same members solved one at a time, and the batched step phase as
    grid-point RK-stage updates per second."""
    import torch
    from piafs_b200 import Batch, Simulation, cases
    tmp = tempfile.mkdtemp(prefix="piafs_bench_ens_")
    try:
        mem = cases.ensemble(tmp, n=members, steps=steps)
        with Batch() as B:        # modules and context warm
            B.add(mem[0]["dir"], 1)
            B.step(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with Batch() as B:
            ids = B.add_many([m["dir"] for m in mem], [steps] * len(mem))
            t1 = time.perf_counter()
            B.step(steps)
            t2 = time.perf_counter()
            for i in ids:
                B.solution(i)
        batched = time.perf_counter() - t0
        t0 = time.perf_counter()
        for m in mem:
            with Simulation(m["dir"]) as sim:
                sim.time_rk(steps)
                sim.solution()
        single = time.perf_counter() - t0
        pts = sum(m["side"] ** 2 for m in mem)
        return {"members": members, "steps": steps, "sides": [min(m["side"] for m in mem), max(m["side"] for m in mem)],
                "batched_solves_per_s": members / batched, "one_at_a_time_solves_per_s": members / single,
                "speedup": single / batched, "step_phase_pt_stage_updates_per_s": 3 * steps * pts / (t2 - t1),
                "precision": "fp64", "full_workload": "bench.py --workload ensemble (256 members, 100 steps)"}
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def slab_bench(a):
    """One 2D photochemical grid decomposed over the N ranks (row slabs, NCCL
    all-to-all exchanges; piafs_b200/slab.py): strong scaling of the default
    workload's grid.  Needs N >= 2 GPUs.  Timed like the replicas: chunks of
    steps from the initial condition, barrier-bracketed, CUDA events on each
    rank's stream, max over ranks."""
    import numpy as np
    import torch
    import torch.distributed as dist
    from piafs_b200.slab import SlabSimulation

    rank, world, barrier = _dist_setup()
    if world < 2:
        sys.exit("bench.py --workload slab decomposes one grid over --gpus N >= 2 ranks")
    tmp = tempfile.mkdtemp(prefix=f"piafs_slab_r{rank}_")
    try:
        a2 = argparse.Namespace(**{**vars(a), "workload": "ns2d_photochem"})
        meta = make_deck(tmp, a2, a.warmup + a.steps)
        sl = SlabSimulation(tmp, precision=a.precision)
        N0, N1 = meta["size"]
        stream = torch.cuda.ExternalStream(sl.stream)
        u0 = sl.state()
        t0 = 0.0

        def chunks(n):
            while n > 0:
                k = min(chunk_steps(max(N0, N1)), n)
                yield k
                n -= k

        for k in chunks(a.warmup):
            sl.set_state(u0, t0)
            sl.step(k)
        total_ms = 0.0
        for k in chunks(a.steps):
            sl.set_state(u0, t0)
            barrier()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sl.step(k)
            e1.record(stream)
            torch.cuda.synchronize()
            barrier()
            total_ms += e0.elapsed_time(e1)
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        units = 3 * N0 * N1 * a.steps
        if rank == 0:
            line = {"metric": "pt-stage updates/s", "value": units / (ms / 1e3), "unit": "pt-stage updates/s",
                    "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps,
                    "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                    "data": "synthetic (seeded deck of the workload's shape)",
                    "config": {"workload": f"ns2d_photochem_crweno5_llf_ssprk3_{N0}x{N1}_slabs{world}",
                               "parallelism": f"row slabs x {world}", "precision": a.precision},
                    "gpu_launches": None}
            print(json.dumps(line))
        sl.close()
        return 0
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def relaunch_under_torchrun(a):
    """--gpus N > 1 started as a plain process: run the same command as N
    ranks (one per GPU) under torch.distributed.run and return its status."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={a.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", os.environ.get("MASTER_PORT", "29533"),
           os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(cmd).returncode


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch_under_torchrun(a)
    if a.impl == "gpu" and world != a.gpus:
        sys.exit(f"bench.py: --gpus {a.gpus} but {world} rank(s) were launched")
    n_gpus = max(world, 1)
    metric = "pt-stage updates/s"

    if a.workload == "ensemble" and a.impl == "gpu":
        return ensemble_bench(a)
    if a.workload == "serving" and a.impl == "gpu":
        return serving_bench(a)
    if a.workload == "slab" and a.impl == "gpu":
        return slab_bench(a)

    if a.impl == "reference":
        if rank != 0:
            return 0
        w, units, cores, kind, sample = run_reference_steps(a, a.steps, a.warmup)
        total = sum(w)
        v = units * len(w) / total
        meta_n = sample_size(a.steps, a.warmup) if a.workload == "ns2d_photochem" else (a.n or 1024)
        line = {"impl": "reference", "metric": metric, "value": v, "unit": metric, "n_gpus": a.gpus,
                "steps": len(w), "warmup": a.warmup, "ms_per_step": 1e3 * total / max(len(w), 1),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded decks of the workload's shape)",
                "config": {"workload": ("ns2d_photochem_crweno5_llf_ssprk3" if a.workload == "ns2d_photochem"
                                        else "euler1d_weno5_roe_ssprk3") + f"_sample_{meta_n}",
                           "sample_of": "2048x2048" if a.workload == "ns2d_photochem" else str(meta_n)},
                "cpu_baseline": {"value": v, "unit": metric, "cores": cores, "kind": kind, "sample": sample},
                "e2e": {"value": v, "unit": metric, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import numpy as np
    import torch
    import piafs_b200
    from piafs_b200 import Simulation

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x):
        if world <= 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    tmp = tempfile.mkdtemp(prefix=f"piafs_bench_r{rank}_")
    try:
        meta = make_deck(tmp, a, a.warmup + a.steps)
        sim = Simulation(tmp, precision=a.precision)
        info = sim.info
        npts = info["dim"][0] * info["dim"][1]
        units_per_step = info["nstages"] * npts
        N = max(info["dim"][0], info["dim"][1])
        stream = torch.cuda.ExternalStream(sim.stream)

        u0, t0 = sim.state(), info["t"]

        def reset():
            sim.set_state(u0, t0)

        # warm-up (also instantiates the CUDA graph of a step)
        done = 0
        while done < a.warmup:
            reset()
            n = min(chunk_steps(N), a.warmup - done)
            sim.time_rk(n)
            done += n
        # timed: K steps in chunks of at most chunk_steps(N) from the initial state,
        # each chunk bracketed by barrier + synchronize, device time summed
        ms = 0.0
        with ClockSampler(local) as clk:
            time.sleep(0.3)
            done = 0
            while done < a.steps:
                n = min(chunk_steps(N), a.steps - done)
                reset()
                barrier()
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                sim.time_rk_async(n)
                e1.record(stream)
                torch.cuda.synchronize()
                barrier()
                ms += e0.elapsed_time(e1)
                done += n
        ms_max = max_over_ranks(ms)
        assert sim.info["singular"] == 0, "zero pivot during the benchmark"
        sol_ok = bool(np.isfinite(sim.solution()).all())
        last_chunk = n
        value = units_per_step * a.steps * n_gpus / (ms_max / 1e3)

        # mixed precision: error against the FP64 path after one full chunk of
        # steps from the same initial state
        err = None
        if a.precision == "mixed":
            last_chunk = chunk_steps(N)
            reset()
            sim.time_rk(last_chunk)
            got = sim.solution()
            with Simulation(tmp, precision="fp64") as ref_sim:
                ref_sim.time_rk(last_chunk)
                ref = ref_sim.solution()
            rms = np.sqrt((ref * ref).mean(axis=0))
            l2 = np.sqrt(((got - ref) ** 2).sum(axis=0) / np.maximum((ref * ref).sum(axis=0), 1e-300))
            linf = np.abs(got - ref).max(axis=0) / np.maximum(np.abs(ref).max(axis=0), 1e-300)
            sig = rms >= 1e-6 * rms.max()
            err = {"vs": "FP64 GPU path, same deck", "steps": last_chunk,
                   "rel_l2_max": float(l2[sig].max()), "rel_linf_max": float(linf[sig].max()),
                   "rel_l2_per_var": [float(x) for x in l2]}

        # dominant kernel: per-phase device time of one RHS evaluation
        phases = sim.profile_rhs(reps=3)
        dom = max(phases, key=phases.get)
        nv = info["nvars"]
        bpu = BYTES_PER_UNIT.get(nv, 3 * nv * 8)
        peaks = {}
        pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.exists(pk):
            peaks = json.load(open(pk))
        peak = peaks.get("hbm_gbs", 6650.0)
        achieved = bpu * npts / (phases[dom] / 1e3) / 1e9
        # DRAM bytes per launch of the dominant kernel from the ncu capture of
        # k_crw_line at 1536^2 (read + write per interior point, scaled by
        # the points processed); known for the FP64 CRWENO5 line solve only
        traffic = None
        if dom.startswith("reconstruct") and a.precision == "fp64" and (a.scheme or "crweno5") == "crweno5" \
                and info["nvars"] in TRAFFIC_PER_POINT:
            traffic = TRAFFIC_PER_POINT[info["nvars"]] * npts
        step_ms = ms_max / a.steps
        path_gbs = bpu * units_per_step / (step_ms / 1e3) / 1e9 / 1.0
        roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": traffic,
                    "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                    "units_per_launch": npts, "bytes_per_unit": bpu,
                    "phase_ms": {k: round(v, 4) for k, v in phases.items()},
                    "path_gbs": path_gbs, "path_frac": path_gbs / peak}

        # end to end through the C ABI with host buffers: H2D of the state,
        # one step, D2H of the state, every step
        ne = max(1, min(a.e2e_steps, a.steps))
        shape = sim.shape_ghosted
        pinned = torch.empty(shape[0] * shape[1], dtype=torch.float64, pin_memory=True)
        uh = pinned.numpy()
        uh[:] = u0
        t = t0
        barrier()
        torch.cuda.synchronize()
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record(stream)
        for _ in range(ne):
            sim.time_rk_host(uh, t)
            t += info["dt"]
        h1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = max_over_ranks(h0.elapsed_time(h1))
        e2e = {"value": units_per_step * ne * n_gpus / (e2e_ms / 1e3), "unit": metric,
               "h2d_bytes_per_step": int(uh.nbytes), "d2h_bytes_per_step": int(uh.nbytes),
               "steps": ne, "ms_per_step": e2e_ms / ne,
               "api": "piafs_gpu_TimeRK_host (pinned host state in, one step, state out)"}
        launches = info["launches_per_step"] * a.steps
        # the mixed-precision and batched-ensemble figures of the same run
        # (rank 0, after the timed regions)
        extras = {}
        if rank == 0 and a.precision == "fp64" and a.workload == "ns2d_photochem" and not a.no_extras:
            try:
                extras["mixed"] = mixed_figure(tmp, a, sim, u0, t0, N, step_ms)
            except Exception as ex:  # reported, not fatal
                extras["mixed"] = {"error": str(ex)[:200]}
        sim.close()
        if rank == 0 and a.workload == "ns2d_photochem" and not a.no_extras:
            try:
                extras["ensemble"] = ensemble_figure()
            except Exception as ex:  # reported, not fatal
                extras["ensemble"] = {"error": str(ex)[:200]}

        base = None
        if rank == 0 and world == 1 and not a.no_cpu_baseline:
            try:
                base = cpu_baseline(a)
            except Exception as ex:  # reported, not fatal
                base = {"value": None, "error": str(ex)[:200]}
        if rank == 0:
            line = {"metric": metric, "value": value, "unit": metric, "n_gpus": n_gpus, "steps": a.steps,
                    "warmup": a.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f64" if a.precision == "fp64" else "f32+f64",
                    "data": "synthetic (seeded decks of the workload's shape)",
                    "config": workload_config(a, meta, n_gpus), "roofline": roofline, "cpu_baseline": base,
                    "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(), "finite": sol_ok,
                    "precision": a.precision}
            if err is not None:
                line["error_vs_fp64"] = err
            line.update(extras)
            print(json.dumps(line))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
