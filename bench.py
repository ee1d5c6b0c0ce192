#!/usr/bin/env python
"""Benchmark: games/s of the batched energy-game solver.

Workload (N=1): the batched configuration -- 4,096 seeded LTSs (states
log-uniform in [20, 5000], 2-16 labels, 1.5-5 transitions per state, tau
p = 0.2), one compare(p, q) game each, minimised and built on the host, all
solved together on the device.  Jobs are taken in seed order, skipping
bisimilar pairs and games above 200,000 positions (gpuequiv_b200/data/
batched_seeds.json lists them).  A step = one solve of the whole batch.

  value        games/s with the games resident in HBM (device-timed solves)
  e2e          games/s through geq_energy_game_run_batch with host buffers
               (upload + solve + download inside the timed region)
  plain_cuda   games/s of one geq_energy_game_run call per game (a sample)
  cpu_baseline the oracle on one host thread (a sample)
  --impl reference: the oracle on all host threads (a sample), same metric.

Under torchrun each rank solves its own batch (different seeds): weak
scaling, no collective on the data path; the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "games/s (batched spectroscopy energy games, bit-exact)"
UNIT = "games/s"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--jobs", type=int, default=4096)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--plain-sample", type=int, default=256)
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (default launch shape)")
    ap.add_argument("--serve-rates", default="1000,5000",
                    help="Poisson arrival rates (req/s) of the serving leg; empty: no serving leg")
    ap.add_argument("--serve-seconds", type=float, default=3.0, help="arrivals per serving rate (s)")
    ap.add_argument("--no-stress", dest="stress", action="store_false", help="skip the stress-game leg")
    ap.add_argument("--solve-only", action="store_true",
                    help="build, upload and solve only (the command profiled with ncu)")
    ap.add_argument("--build-only", action="store_true",
                    help="one device GameBuild of the batch's minimised LTSs only (profiled with ncu)")
    ap.add_argument("--no-graph", action="store_true",
                    help="with --build-only: levels as plain launches (ncu does not profile kernels of a graph "
                         "with conditional nodes)")
    return ap.parse_args()


# ---- distributed plumbing -------------------------------------------------------
class Dist:
    """One process per GPU.  NCCL between GPUs; `backend="gloo"` runs the same
    host logic on CPU ranks (the multi-rank tests)."""

    def __init__(self, backend: str | None = None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        self.device = "cpu"
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            backend = backend or "nccl"
            if backend == "nccl":
                torch.cuda.set_device(self.local_rank)
                self.device = "cuda"
                dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                        device_id=torch.device("cuda", self.local_rank))
            else:
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = dist

    def barrier(self):
        if self.pg:
            import torch
            t = torch.zeros(1, device=self.device)
            self.pg.all_reduce(t)
            if self.device == "cuda":
                torch.cuda.synchronize()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.pg.all_reduce(t)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---- clocks ---------------------------------------------------------------------
class Clocks:
    """nvidia-smi sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(gpu)], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except subprocess.TimeoutExpired:
                self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---- workload -------------------------------------------------------------------
_SYNTH = None


def synth_mod():
    """gpuequiv_b200/synth.py loaded by path: the generators need only numpy,
    and the reference arm must not load libgeq."""
    global _SYNTH
    if _SYNTH is None:
        import importlib.util
        spec = importlib.util.spec_from_file_location("geq_synth", os.path.join(ROOT, "gpuequiv_b200", "synth.py"))
        _SYNTH = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(_SYNTH)
    return _SYNTH


def batched_seeds(n_jobs: int, rank: int):
    synth = synth_mod()
    if rank == 0:
        m = synth.batched_manifest()
        rows = m["jobs"][:n_jobs]
        if len(rows) == n_jobs:
            return [r[0] for r in rows], rows
    jobs = synth.select_batched_jobs(n_jobs, first_seed=1_000_000 * rank)
    rows = [[j["seed"], int(j["build"].game.n_vertices()), int(j["build"].game.n_edges())] for j in jobs]
    return [r[0] for r in rows], rows


def build_games_ours(seeds):
    """Minimise + build every job with libgeq's host builder (not timed)."""
    from concurrent.futures import ThreadPoolExecutor

    import gpuequiv_b200 as geq
    synth = synth_mod()

    def one(seed):
        src, dst, lab, p, q = synth.batched_lts(seed)
        lts = geq.TransitionSystem.from_arrays(src, dst, lab)
        red, mp = lts.bisimilar_minimize()
        b = geq.GameBuild.compare(red, int(mp[p]), int(mp[q]))
        return b.game

    with ThreadPoolExecutor(max_workers=min(32, os.cpu_count() or 4)) as ex:
        return list(ex.map(one, seeds))


def build_games_oracle(seeds):
    """The same jobs built by the oracle's own restatement of GameBuild."""
    from oracle import ora
    synth = synth_mod()
    games = []
    for seed in seeds:
        src, dst, lab, p, q = synth.batched_lts(seed)
        lts = ora.Lts.from_arrays(src, dst, lab)
        red, mp = lts.bisimilar_minimize()
        b = ora.Build.compare(red, int(mp[p]), int(mp[q]))
        games.append((b.row, b.col, b.wt, b.attacker))
    return games


def sample_indices(n: int, k: int):
    return list(range(0, n, max(1, n // k)))[:k]


def oracle_rate(games, threads: int, budget_s: float):
    """Solve games with the oracle until the budget is spent; games/s."""
    from oracle import ora
    done, t0 = 0, time.perf_counter()
    chunk = max(1, threads * 4)
    while done < len(games):
        ora.run_games_parallel(games[done:done + chunk], threads=threads)
        done = min(len(games), done + chunk)
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return done / dt, done, dt


def peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def profile_traffic_ratio():
    """DRAM bytes per algorithmic byte of k_round, from the committed ncu
    summary (all round launches of a smaller case of the same workload)."""
    p = os.path.join(ROOT, "profiles", "k_round_batched.md")
    try:
        with open(p) as f:
            for line in f:
                if line.strip().startswith("dram_per_algorithmic_byte:"):
                    return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


def run_serving(ctx, graphs, lam: float, seconds: float, seed: int, queries=False) -> dict:
    """Poisson arrivals of single requests (drawn from `graphs`) into the
    serving loop; latency = submit -> result in the caller's hands.  With
    `queries`, the items are (lts, p, q) equivalence queries (minimised, built
    and solved on the device), else game graphs."""
    import queue
    import threading

    from gpuequiv_b200.serving import Server
    rng = np.random.default_rng(seed)
    n = max(1, int(lam * seconds))
    arrivals = np.cumsum(rng.exponential(1.0 / lam, n))
    pick = rng.integers(0, len(graphs), n)
    t_sub = np.zeros(n)
    t_done = np.zeros(n)
    with Server(ctx) as srv:
        submit = (lambda item: srv.submit_compare(*item)) if queries else srv.submit
        # warm the pipelines (CUDA graphs, device and host pools): single
        # requests, then a burst
        for g in graphs[:32]:
            srv.poll(submit(g))
        for t in [submit(g) for g in graphs[:512]]:
            srv.poll(t)
        q: "queue.Queue" = queue.Queue()

        def poller():
            while True:
                item = q.get()
                if item is None:
                    return
                i, t = item
                srv.poll(t)
                t_done[i] = time.perf_counter()

        pollers = [threading.Thread(target=poller) for _ in range(4)]
        for th in pollers:
            th.start()
        st0 = srv.stats()
        t0 = time.perf_counter()
        for i in range(n):
            wait = t0 + arrivals[i] - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
            t_sub[i] = time.perf_counter()
            q.put((i, submit(graphs[pick[i]])))
        for _ in pollers:
            q.put(None)
        for th in pollers:
            th.join()
        st = srv.stats()
    lat = (t_done - t_sub) * 1e3
    span = t_done.max() - t0
    batches = st["batches"] - st0["batches"]
    return {"lambda_req_s": lam, "requests": n, "seconds": round(float(span), 3),
            "throughput_games_s": n / span, "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
            "batches": int(batches), "mean_batch": (st["games_in_batches"] - st0["games_in_batches"]) / max(1, batches)}


# ---- arms -----------------------------------------------------------------------
def run_lts_pipeline(ctx, seeds, graphs, args, d: Dist) -> dict:
    """compare_batch over the batch's LTSs: the whole LTS -> energies path
    (minimisation and GameBuild on the device, batched solve, start-position
    energies read back), beside the device GameBuild alone and the host
    GameBuild of the same minimised LTSs on all host cores."""
    from concurrent.futures import ThreadPoolExecutor

    import gpuequiv_b200 as geq
    synth = synth_mod()
    jobs = []
    for seed in seeds:
        src, dst, lab, p, q = synth.batched_lts(seed)
        jobs.append((geq.TransitionSystem.from_arrays(src, dst, lab), int(p), int(q)))
    # the start energies agree with the resident solve's (first 64 games)
    first = geq.compare_batch(jobs[:64], context=ctx)
    offs, data, _ = geq.run_batch_raw(graphs[:64], ctx, geq.c_views(graphs[:64]))
    for k in range(len(first)):
        ref = sorted(int(x) for x in data[k][offs[k][0]:offs[k][1]].reshape(-1))
        assert sorted(int(x) for x in np.asarray(first[k].array).reshape(-1)) == ref, f"job {k}"
    geq.compare_batch(jobs, context=ctx)  # warm-up
    d.barrier()
    times = []
    for _ in range(max(1, min(args.steps, 3))):
        t = time.perf_counter()
        geq.compare_batch(jobs, context=ctx)
        times.append(time.perf_counter() - t)
    pipe_s = d.max(float(np.median(times)))
    # the two builders alone, on the minimised LTSs
    reds = []
    for lts, p, q in jobs:
        red, mp = lts.bisimilar_minimize()
        reds.append((red, int(mp[p]), int(mp[q])))
    b = geq.GameBatch(reds, context=ctx)
    dev_build = []
    for _ in range(3):
        b = geq.GameBatch(reds, context=ctx)
        dev_build.append(b.stats["upload_ms"] + b.stats["build_ms"])
    threads = os.cpu_count() or 4
    t = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(lambda j: geq.GameBuild.compare(*j), reds))
    host_build_ms = (time.perf_counter() - t) * 1e3
    # the plain form: one compare() call per query (every 32nd job)
    sample = jobs[::32]
    for j in sample[:8]:
        geq.compare_batch([j], context=ctx)
    t = time.perf_counter()
    for j in sample:
        geq.compare_batch([j], context=ctx)
    plain_q = len(sample) / (time.perf_counter() - t)
    return jobs, {"workload": "compare_batch over the same 4096 LTSs (unminimised): device minimisation, device GameBuild, "
                        "batched solve, start energies read back",
            "games_s": d.sum(len(jobs)) / pipe_s, "ms_per_step": pipe_s * 1e3,
            "device_build_ms": float(np.median(dev_build)), "build_levels": b.stats["levels"],
            "build_kernel_launches": b.stats["kernel_launches"],
            "host_build_ms_all_cores": host_build_ms, "host_threads": threads,
            "plain_per_query": {"value": plain_q, "unit": UNIT,
                                "sample": f"{len(sample)} jobs (every 32nd), one compare() call each"},
            "batched_vs_plain_per_query": (d.sum(len(jobs)) / pipe_s) / plain_q if plain_q else None}


def run_reference(args, d: Dist):
    if d.rank != 0:
        return
    seeds, rows = batched_seeds(args.jobs, 0)
    idx = sample_indices(len(seeds), 512)
    games = build_games_oracle([seeds[i] for i in idx])
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        oracle_rate(games[:threads], threads, 5.0)
    rates = []
    for _ in range(args.steps):
        r, n, dt = oracle_rate(games, threads, max(5.0, 60.0 / max(args.steps, 1)))
        rates.append((r, n, dt))
    value = float(np.median([r[0] for r in rates]))
    sample = (f"{rates[0][1]} of {len(games)} games (every {max(1, len(seeds) // 512)}th job of the "
              f"{len(seeds)}-job batch) per step, oracle EnergyGame::run on {threads} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.median([r[2] for r in rates]) * 1e3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"batched: {len(seeds)} seeded LTS compare(p,q) spectroscopy games"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_build_only(args, d: Dist):
    """One device GameBuild of the batch (GameBuild::compare of every job's
    minimised LTS), nothing else on the device: the command profiled for the
    builder's launch list."""
    from concurrent.futures import ThreadPoolExecutor

    import gpuequiv_b200 as geq
    synth = synth_mod()
    seeds, _ = batched_seeds(args.jobs, d.rank)

    def prep(seed):
        src, dst, lab, p, q = synth.batched_lts(seed)
        red, mp = geq.TransitionSystem.from_arrays(src, dst, lab).bisimilar_minimize()
        return red, int(mp[p]), int(mp[q])

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        jobs = list(ex.map(prep, seeds))
    ctx = geq.Context(d.local_rank)
    if args.no_graph:
        from gpuequiv_b200._lib import TUNE_NO_GRAPH
        ctx.set_tuning(flags=TUNE_NO_GRAPH)
    b = geq.GameBatch(jobs, context=ctx)
    if d.rank == 0:
        print(json.dumps({"build_only": True, "jobs": len(jobs), "stats": b.stats}), flush=True)
    del b
    ctx.close()


def run_ours(args, d: Dist):
    import gpuequiv_b200 as geq
    from gpuequiv_b200._lib import TUNE_PROFILE
    if args.build_only:
        return run_build_only(args, d)
    ctx = geq.Context(d.local_rank)
    seeds, rows = batched_seeds(args.jobs, d.rank)
    t = time.perf_counter()
    graphs = build_games_ours(seeds)
    build_s = time.perf_counter() - t
    pos = sum(g.n_vertices() for g in graphs)
    edges = sum(g.n_edges() for g in graphs)
    assert [g.n_vertices() for g in graphs] == [r[1] for r in rows], "game sizes differ from the manifest"
    in_bytes = sum(g.row_offsets.nbytes + g.column_indices.nbytes + g.weights.array.nbytes + g.attacker_pos.nbytes
                   for g in graphs)

    # ---- value: games resident in HBM ----
    dg = geq.DeviceGames(graphs, ctx)
    tune = None
    if not args.no_tune:
        from gpuequiv_b200.autotune import autotune
        tune = autotune(dg, ctx, f"batched-{len(graphs)}", use_cache=False)
    for _ in range(args.warmup):
        dg.solve()
    if args.solve_only:
        for _ in range(args.steps):
            st = dg.solve()
        if d.rank == 0:
            print(json.dumps({"solve_only": True, "games": len(graphs), "positions": pos, "edges": edges,
                              "stats": st}), flush=True)
        dg.close()
        ctx.close()
        return
    d.barrier()
    clocks = Clocks(d.local_rank)
    dev_ms, launches, st_last = 0.0, 0, None
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st_last = dg.solve()
        dev_ms += st_last["device_ms"]
        launches += st_last["kernel_launches"]
    wall_ms = (time.perf_counter() - t0) * 1e3
    ck = clocks.stop()
    d.barrier()
    step_ms = d.max(dev_ms / args.steps)
    total_games = d.sum(len(graphs))
    value = total_games / (step_ms / 1e3)

    # ---- roofline of the round kernel (one profiled solve, not timed) ----
    ctx.set_tuning(flags=TUNE_PROFILE)
    st_prof = dg.solve()
    ctx.set_tuning(flags=0)
    dg.close()
    peak, peak_kind = peak_hbm()
    k_ms = st_prof["round_kernel_ms"]
    k_launch = max(1, st_prof["round_kernel_launches"])
    achieved = st_prof["algorithmic_bytes"] / (k_ms / 1e3) / 1e9 if k_ms > 0 else None
    ratio = profile_traffic_ratio()
    alg_per_launch = st_prof["algorithmic_bytes"] / k_launch
    traffic = ratio * alg_per_launch if ratio else None

    # ---- e2e: host buffers through the C ABI (geq_energy_game_run_batch) ----
    views = geq.c_views(graphs)
    for _ in range(max(1, args.warmup // 2)):
        offs, data, _ = geq.run_batch_raw(graphs, ctx, views)
    out_bytes = sum(o.nbytes for o in offs) + sum(x.nbytes for x in data)  # offsets + energies read back
    del offs, data
    d.barrier()
    e2e_t = []
    for _ in range(args.steps):
        t = time.perf_counter()
        geq.run_batch_raw(graphs, ctx, views)
        e2e_t.append(time.perf_counter() - t)
    e2e_s = d.max(float(np.median(e2e_t)))
    e2e = total_games / e2e_s

    # ---- LTS -> verdict: compare_batch from the unminimised LTSs (host
    # minimisation, games built on the device, solved, start energies back) ----
    lts_jobs, lts_pipe = run_lts_pipeline(ctx, seeds, graphs, args, d)

    # ---- plain CUDA: one call per game (sample) ----
    idx = sample_indices(len(graphs), args.plain_sample)
    pviews = [geq.c_views([graphs[i]]) for i in idx]
    for i in range(len(idx)):  # warm-up pass: the pools hold every block size of the sample
        geq.run_batch_raw([graphs[idx[i]]], ctx, pviews[i])
    t = time.perf_counter()
    for i in range(len(idx)):
        geq.run_batch_raw([graphs[idx[i]]], ctx, pviews[i])
    plain_s = time.perf_counter() - t
    plain_rate = len(idx) / plain_s  # every k-th job: the batch's size mix

    # ---- serving loop: Poisson arrivals of single games (not part of value) ----
    serving = []
    rates = [float(x) for x in args.serve_rates.split(",") if x.strip()]
    for k, lam in enumerate(rates):
        serving.append(run_serving(ctx, graphs, lam, args.serve_seconds, seed=100 + k + 1000 * d.rank))
    # the same arrivals as equivalence queries on the LTSs themselves
    serving_q = []
    for k, lam in enumerate(rates):
        serving_q.append(run_serving(ctx, lts_jobs, lam, args.serve_seconds, seed=100 + k + 1000 * d.rank,
                                     queries=True))

    # ---- stress configuration: one 2M-position / 10M-edge game, resident ----
    stress = None
    if args.stress:
        srow, scol, swt, satt = synth_mod().stress_game()
        sg = geq.GameGraph.from_csr(srow, scol, swt, satt, geq.EnergyConf.STANDARD)
        sdg = geq.DeviceGames([sg], ctx)
        for _ in range(2):
            sdg.solve()
        sts = [sdg.solve() for _ in range(3)]
        sdg.close()
        sms = float(np.median([x["device_ms"] for x in sts]))
        stress = {"workload": "stress: 2,000,000 positions (60 % attackers), 10,000,000 edges, seed 2, standard reach",
                  "solve_ms": sms, "edges_relaxed": sts[0]["edges_relaxed"],
                  "positions_computed": sts[0]["positions_computed"], "rounds": sts[0]["rounds"],
                  "edges_relaxed_per_s": sts[0]["edges_relaxed"] / (sms / 1e3)}

    # ---- CPU baseline: the oracle on one host thread (rank 0, N=1) ----
    cpu = None
    if d.rank == 0 and d.world == 1:
        cidx = sample_indices(len(seeds), 256)
        cg = build_games_oracle([seeds[i] for i in cidx])
        r, n, dt = oracle_rate(cg, 1, args.cpu_seconds)
        cpu = {"value": r, "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{n} games (every {max(1, len(seeds) // 256)}th job of the batch, in order) in {dt:.1f} s, "
                         f"oracle EnergyGame::run, 1 thread"}

    if d.rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": d.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": {
                "workload": f"batched: {len(graphs)} seeded LTS compare(p,q) spectroscopy games per GPU "
                            f"(states log-uniform 20-5000, 2-16 labels, 1.5-5 transitions/state; games <= 200k positions)",
                "games_per_gpu": len(graphs), "positions_per_gpu": pos, "edges_per_gpu": edges,
                "host_build_s": round(build_s, 2),
                "l2": f"inputs larger than L2 ({in_bytes / 1e6:.0f} MB of game graph per GPU)",
                "parallelism": f"replicas x{d.world}",
            },
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "traffic_source": "ncu DRAM bytes per algorithmic byte of all round-kernel launches (k_round + "
                                           "k_round_big) of the 1024-job case (profiles/k_round_batched.md) x "
                                           "algorithmic bytes per full-size round",
                         "algorithmic_bytes_per_launch": alg_per_launch,
                         "kernel": "k_round + k_round_big (one round)", "peak_kind": peak_kind,
                         "algorithmic_bytes_per_solve": st_prof["algorithmic_bytes"],
                         "round_kernel_ms_per_solve": k_ms, "round_kernel_launches": k_launch},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(in_bytes),
                    "d2h_bytes_per_step": int(out_bytes)},
            "plain_cuda": {"value": plain_rate, "unit": UNIT, "sample": f"{len(idx)} games (every "
                           f"{max(1, len(graphs) // len(idx))}th job), one geq_energy_game_run call each"},
            "batched_vs_plain": value / plain_rate if plain_rate else None,
            "lts_pipeline": lts_pipe,
            "stress": stress,
            "serving": {"workload": "Poisson arrivals of single compare(p,q) games drawn from this batch "
                                    "(LTS 20-5000 states), geq_server with 2 pipelines, 150 GB admission budget",
                        "runs": serving,
                        "queries": {"workload": "the same Poisson arrivals as compare(p, q) queries on the batch's "
                                                "unminimised LTSs (geq_server_submit_compare: minimisation, "
                                                "GameBuild and solve on the device)", "runs": serving_q}},
            "gpu_launches": int(launches),
            "clocks": ck,
            "solve_stats": {k: st_last[k] for k in ("rounds", "positions_computed", "edges_relaxed",
                                                     "algorithmic_bytes", "arena_compactions")},
            "wall_ms_per_step": wall_ms / args.steps,
            "tuning": ctx.tuning(),
            "autotune": tune,
        }
        print(json.dumps(line), flush=True)
    ctx.close()


def main():
    args = parse()
    d = Dist()
    try:
        if args.impl == "reference":
            run_reference(args, d)
        else:
            run_ours(args, d)
    finally:
        d.close()


if __name__ == "__main__":
    main()
