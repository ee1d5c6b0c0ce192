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


_T0 = time.perf_counter()


def progress(msg: str) -> None:
    """One line of progress on stderr (the JSON result line goes to stdout)."""
    print(f"[bench {time.perf_counter() - _T0:7.1f} s] {msg}", file=sys.stderr, flush=True)


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
    ap.add_argument("--serve-rates", default="5000,10000",
                    help="Poisson arrival rates (req/s) of the game-request serving leg; empty: none")
    ap.add_argument("--query-rates", default="200,1000,5000",
                    help="Poisson arrival rates (req/s) of the serving configuration (equivalence queries on LTSs "
                         "of 20-20,000 states); empty: none")
    ap.add_argument("--serve-seconds", type=float, default=10.0, help="arrivals per serving rate (s)")
    ap.add_argument("--serve-pipelines", type=int, default=0, help="serving pipelines (0: the library default)")
    ap.add_argument("--saturation-seconds", type=float, default=6.0,
                    help="closed-loop saturation run of each serving leg (s); 0: none")
    ap.add_argument("--query-bound", type=int, default=200_000,
                    help="position bound of a served query's game (larger games are refused)")
    ap.add_argument("--query-pool", type=int, default=2048, help="distinct queries the arrivals draw from")
    ap.add_argument("--large-states", type=int, default=16000,
                    help="states of the single-LTS equivalences() leg (the large generator; 0: none)")
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
    """nvidia-smi sampled every 50 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.skip = 0
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "50", "-i", str(gpu)], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def start(self) -> None:
        """Wait (at most 2 s) until the sampler runs; samples taken before
        this call are not counted."""
        t_end = time.perf_counter() + 2.0
        while self.p and time.perf_counter() < t_end:
            with open(self.f.name) as g:
                n = sum(1 for _ in g)
            if n:
                self.skip = n
                return
            time.sleep(0.02)

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
        for line in self.f.read().splitlines()[self.skip:]:
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
        b = ora.Build.compare(red, int(mp[p]), int(mp[q]), positions=False)
        games.append((b.row, b.col, b.wt, b.attacker))
    return games


def canonical(offsets, data):
    """Every position's list sorted: (offsets, data) ordered by (position, word)."""
    o = np.asarray(offsets, np.int64)
    dd = np.asarray(data, np.uint32)
    seg = np.repeat(np.arange(len(o) - 1), np.diff(o))
    return o, dd[np.lexsort((dd, seg))]


def sample_indices(n: int, k: int):
    return list(range(0, n, max(1, n // k)))[:k]


def build_games_oracle_parallel(seeds, threads: int):
    """build_games_oracle on host threads (the oracle's calls release the GIL)."""
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, threads)) as ex:
        return [g for part in ex.map(build_games_oracle, [[s] for s in seeds]) for g in part]


def oracle_solve(games, threads: int):
    """One oracle solve of every game: `threads` threads share one work
    counter, largest games first.  Returns (games/s, seconds, solutions)."""
    from oracle import ora
    t0 = time.perf_counter()
    sols = ora.solve_games(games, threads=threads, largest_first=True)
    dt = time.perf_counter() - t0
    return len(games) / dt, dt, sols


def workload_config(rows, world: int) -> dict:
    """The `config` object of both arms (same workload, same keys)."""
    pos = sum(r[1] for r in rows)
    edges = sum(r[2] for r in rows)
    in_bytes = sum(4 * (r[1] + 1) + 8 * r[2] + r[1] for r in rows)  # row, col, wt, attacker flags
    return {
        "workload": f"batched: {len(rows)} seeded LTS compare(p,q) spectroscopy games per GPU "
                    f"(states log-uniform 20-5000, 2-16 labels, 1.5-5 transitions/state; games <= 200k positions)",
        "games_per_gpu": len(rows), "positions_per_gpu": int(pos), "edges_per_gpu": int(edges),
        "l2": f"inputs larger than L2 ({in_bytes / 1e6:.0f} MB of game graph per GPU)",
        "parallelism": f"replicas x{world}",
    }


# DRAM bytes per algorithmic byte of the round kernels (k_round + k_round_big):
# dram__bytes_read.sum + dram__bytes_write.sum over all their launches in one
# ncu capture of the 1,024-job batch (--solve-only --jobs 1024), divided by
# the algorithmic bytes those launches counted.  Traffic grows with the work
# of a launch, so the full-size figure is this ratio x its algorithmic bytes.
DRAM_PER_ALGORITHMIC_BYTE = 1.61


def peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


class LoadApi:
    """ctypes mirror of the native load driver's callback table
    (gpuequiv_b200/csrc/loadgen.cpp: geq_load_api, geq_load_server)."""
    import ctypes as C
    SUBMIT = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint64))
    POLL = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.c_int32, C.POINTER(C.c_uint64), C.POINTER(C.c_void_p))
    FREE = C.CFUNCTYPE(None, C.c_void_p)

    class Api(C.Structure):
        pass

    class Server(C.Structure):
        pass


_LOADGEN = []


def _loadgen():
    import ctypes as C
    if _LOADGEN:
        return _LOADGEN[0]
    path = os.path.join(ROOT, "gpuequiv_b200", "libgeq_load.so")
    ll = C.CDLL(path)
    LoadApi.Api._fields_ = [("ctx", C.c_void_p), ("submit", LoadApi.SUBMIT), ("poll_any", LoadApi.POLL),
                            ("free_answer", LoadApi.FREE)]
    LoadApi.Server._fields_ = [("server", C.c_void_p), ("games", C.c_void_p), ("game_stride", C.c_size_t),
                               ("lts", C.POINTER(C.c_void_p)), ("p", C.POINTER(C.c_uint32)),
                               ("q", C.POINTER(C.c_uint32)), ("server_submit", C.c_void_p),
                               ("server_submit_compare", C.c_void_p), ("server_poll_any", C.c_void_p),
                               ("solution_free", C.c_void_p)]
    ll.geq_load_server_api.argtypes = [C.POINTER(LoadApi.Server), C.POINTER(LoadApi.Api)]
    ll.geq_load_server_api.restype = None
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int32)
    u32p = C.POINTER(C.c_uint32)
    ll.geq_load_open.argtypes = [C.POINTER(LoadApi.Api), u32p, dp, C.c_uint64, C.c_uint32, C.c_uint32, C.c_double,
                                 dp, ip, dp]
    ll.geq_load_open.restype = C.c_int64
    ll.geq_load_closed.argtypes = [C.POINTER(LoadApi.Api), u32p, C.c_uint32, C.c_uint32, C.c_double, C.c_uint64,
                                   C.c_uint32, C.c_uint32, C.c_uint64, C.c_double, dp, ip,
                                   C.POINTER(C.c_uint64), dp]
    ll.geq_load_closed.restype = C.c_int64
    _LOADGEN.append(ll)
    return ll


class Load:
    """Drives a geq_server through the C ABI from native threads (the load
    driver gpuequiv_b200/csrc/loadgen.cpp, built as libgeq_load.so): arrival
    i submits item pick[i] (a game view or an (lts, p, q) query) at its
    arrival time (open loop), or `outstanding` requests are kept in flight
    (closed loop).  Finished requests are taken from the server's completion
    queue (geq_server_poll_any) in the order they finish.  Latency = submit
    -> the request's solution in the caller's hands.  A Python driver was
    measured to cap the closed loop near 30k requests/s by itself (the
    interpreter lock around every submit and poll); this one does not.
    `api`: a LoadApi.Api to drive instead of the server (tests)."""

    def __init__(self, srv, items, queries: bool, threads: int = 4, drain_s: float = 60.0, api=None):
        import ctypes as C
        self.ll = _loadgen()
        self.threads, self.drain_s = threads, drain_s
        if api is None:
            from gpuequiv_b200._lib import geq_game_graph, lib
            ls = LoadApi.Server()
            ls.server = srv.h.value if hasattr(srv.h, "value") else srv.h
            addr = lambda f: C.cast(f, C.c_void_p).value  # noqa: E731
            if queries:
                self._lts = (C.c_void_p * len(items))(*[lts.h.value for lts, _, _ in items])
                self._p = np.ascontiguousarray([p for _, p, _ in items], np.uint32)
                self._q = np.ascontiguousarray([q for _, _, q in items], np.uint32)
                ls.lts = self._lts
                ls.p = self._p.ctypes.data_as(C.POINTER(C.c_uint32))
                ls.q = self._q.ctypes.data_as(C.POINTER(C.c_uint32))
            else:
                ls.games = C.addressof(items)  # a ctypes array of geq_game_graph
                ls.game_stride = C.sizeof(geq_game_graph)
            ls.server_submit = addr(lib.geq_server_submit)
            ls.server_submit_compare = addr(lib.geq_server_submit_compare)
            ls.server_poll_any = addr(lib.geq_server_poll_any)
            ls.solution_free = addr(lib.geq_solution_free)
            self._ls, self._items = ls, items
            api = LoadApi.Api()
            self.ll.geq_load_server_api(C.byref(ls), C.byref(api))
        self.api = api

    def _threads(self):
        return max(1, self.threads // 2), max(1, self.threads // 2)

    # the closed loop's submitters: a submit copies its game (a few hundred
    # KB) into the server; two threads cannot keep 8,192 requests in flight
    # (measured: 37k games/s with a shallow queue), eight can
    CLOSED_SUBMIT_THREADS = 8

    def open_loop(self, arrivals, pick):
        import ctypes as C
        n = len(arrivals)
        arr = np.ascontiguousarray(arrivals, np.float64)
        pk = np.ascontiguousarray(pick, np.uint32)
        lat = np.zeros(max(n, 1), np.float64)
        st = np.full(max(n, 1), -1, np.int32)
        span = C.c_double(0.0)
        ns, npoll = self._threads()
        r = self.ll.geq_load_open(C.byref(self.api), pk.ctypes.data_as(C.POINTER(C.c_uint32)),
                                  arr.ctypes.data_as(C.POINTER(C.c_double)), n, ns, npoll, self.drain_s,
                                  lat.ctypes.data_as(C.POINTER(C.c_double)), st.ctypes.data_as(C.POINTER(C.c_int32)),
                                  C.byref(span))
        if r < 0:
            raise RuntimeError("load driver: invalid arguments")
        return lat[:n], st[:n], span.value

    def closed_loop(self, pick, outstanding: int, seconds: float, cap_rate: float = 400_000.0):
        import ctypes as C
        pk = np.ascontiguousarray(pick, np.uint32)
        cap = int(seconds * cap_rate) + outstanding + 1024
        lat = np.zeros(cap, np.float64)
        st = np.full(cap, -1, np.int32)
        nsub = C.c_uint64(0)
        span = C.c_double(0.0)
        ns, npoll = max(self._threads()[0], self.CLOSED_SUBMIT_THREADS), self._threads()[1]
        r = self.ll.geq_load_closed(C.byref(self.api), pk.ctypes.data_as(C.POINTER(C.c_uint32)), len(pk),
                                    outstanding, seconds, cap, ns, npoll, 1, self.drain_s,
                                    lat.ctypes.data_as(C.POINTER(C.c_double)),
                                    st.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(nsub), C.byref(span))
        if r < 0:
            raise RuntimeError("load driver: invalid arguments")
        n = int(nsub.value)
        return lat[:n], st[:n], span.value


def _lat_summary(lat_ms, status, span_s):
    fin = status >= 0
    ok = status == 0
    refused = int((status == 2).sum())  # GEQ_ERR_OUT_OF_MEMORY: the game exceeds the position bound
    unfinished = int((~fin).sum())      # still running when the drain deadline passed
    failed = int(fin.sum() - ok.sum()) - refused
    l = lat_ms[ok[:len(lat_ms)]] if ok.any() else np.zeros(1)
    return {"requests": int(len(status)), "served": int(ok.sum()), "refused": refused, "failed": failed,
            "unfinished_at_deadline": unfinished,
            "refusal_rate": refused / max(1, len(status)), "seconds": round(float(span_s), 3),
            "throughput_games_s": float(ok.sum() / span_s) if span_s > 0 else None,
            "p50_ms": float(np.percentile(l, 50)), "p99_ms": float(np.percentile(l, 99)), "mean_ms": float(l.mean())}


def run_serving(ctx, items, queries: bool, rates, seconds: float, seed: int, saturation_s: float,
                max_game_positions: int = 0, outstanding: int = 8192, saturation_items=None,
                n_pipelines: int = 0) -> dict:
    """One server: open-loop Poisson arrivals at each rate, then a closed-loop
    saturation run (`outstanding` requests kept in flight) over
    `saturation_items` (default: all items)."""
    from gpuequiv_b200.serving import Server
    rng = np.random.default_rng(seed)
    out = {"runs": [], "saturation": None}
    with Server(ctx, n_pipelines=n_pipelines, max_game_positions=max_game_positions) as srv:
        load = Load(srv, items, queries)
        # warm the pipelines (CUDA graphs, device and host pools): single
        # requests, then a burst
        warm = np.arange(min(len(items), 512))
        load.open_loop(np.zeros(min(32, len(warm))), warm[:32])
        load.open_loop(np.zeros(len(warm)), warm)
        if saturation_s > 0:  # the page-locked input pool up to the saturation run's depth
            load.closed_loop(np.arange(len(items)) if saturation_items is None
                             else np.asarray(saturation_items, np.int64), outstanding, 3.0)
        for lam in rates:
            n = max(1, int(rng.poisson(lam * seconds)))
            arrivals = np.sort(rng.uniform(0, seconds, n))
            pick = rng.integers(0, len(items), n)
            progress(f"  open loop {lam:.0f} req/s, {n} requests")
            st0 = srv.stats()
            lat, status, span = load.open_loop(arrivals, pick)
            st = srv.stats()
            r = _lat_summary(lat, status, span)
            batches = st["batches"] - st0["batches"]
            r.update({"lambda_req_s": lam, "batches": int(batches),
                      "mean_batch": (st["games_in_batches"] - st0["games_in_batches"]) / max(1, batches),
                      "pipeline_thread_ms": {k: round(st[k] - st0[k], 1) for k in ("admit_ms", "step_ms", "retire_ms")}})
            out["runs"].append(r)
        if saturation_s > 0:
            pick = np.arange(len(items)) if saturation_items is None else np.asarray(saturation_items, np.int64)
            progress(f"  closed loop, {outstanding} in flight")
            st0 = srv.stats()
            lat, status, span = load.closed_loop(pick, outstanding, saturation_s)
            st = srv.stats()
            r = _lat_summary(lat, status, span)
            batches = st["batches"] - st0["batches"]
            r.update({"outstanding": outstanding, "batches": int(batches),
                      "mean_batch": (st["games_in_batches"] - st0["games_in_batches"]) / max(1, batches),
                      "pipeline_thread_ms": {k: round(st[k] - st0[k], 1) for k in ("admit_ms", "step_ms", "retire_ms")}})
            out["saturation"] = r
    return out


def within_bound(job, bound: int) -> bool:
    """The game of compare(p, q) (after minimisation) has at most `bound`
    positions (host GameBuild with the bound)."""
    import gpuequiv_b200 as geq
    lts, p, q = job
    red, mp = lts.bisimilar_minimize()
    if mp[p] == mp[q]:
        return True
    try:
        geq.GameBuild.compare_bounded(red, int(mp[p]), int(mp[q]), bound)
        return True
    except geq.GeqError:
        return False


def serving_queries(n_pool: int, seed: int = 7):
    """A pool of equivalence queries with the serving configuration's
    distribution: each a seeded LTS of log-uniform 20-20,000 states (other
    parameters as the batched configuration) and one pair p != q."""
    import gpuequiv_b200 as geq
    synth = synth_mod()
    _, seeds = synth.serving_trace(seed, n_pool, 1.0)
    out = []
    for s in seeds[:n_pool]:
        src, dst, lab, p, q = synth.batched_lts(int(s), smax=20_000)
        out.append((geq.TransitionSystem.from_arrays(src, dst, lab), int(p), int(q)))
    return out


def run_small(ctx, seeds, check: bool) -> dict:
    """The small configuration: TransitionSystem::equivalences() (minimise ->
    compare_all game -> solve -> verdicts) of seeded 40-state LTSs, one call
    per LTS.  With `check` (the CPU baseline leg) the oracle computes the same
    equivalences on one thread: its time is the baseline, and every start
    pair's energies and the 13 standard relations are compared."""
    import gpuequiv_b200 as geq
    synth = synth_mod()
    systems = [synth.small_lts(s) for s in seeds]
    ltss = [geq.TransitionSystem.from_arrays(*x) for x in systems]
    for lts in ltss[:5]:
        lts.equivalences(ctx)
    t = time.perf_counter()
    eqs = [lts.equivalences(ctx) for lts in ltss]
    dt = time.perf_counter() - t
    out = {"workload": f"small: seeds {seeds[0]}..{seeds[-1]}, 40 states, 4 labels, 120 transitions (tau p 0.2), "
                       f"equivalences() per LTS (minimisation, compare_all game, solve, verdicts)",
           "games_s": len(ltss) / dt, "ms_per_game": dt / len(ltss) * 1e3}
    if not check:
        return out
    from oracle import ora
    t = time.perf_counter()
    oeqs = [ora.equivalences(ora.Lts.from_arrays(*x)) for x in systems]
    odt = time.perf_counter() - t
    names = geq.std_equivalences.names()
    bad = []
    for k, (eq, oeq, lts) in enumerate(zip(eqs, oeqs, ltss)):
        n = lts.n_vertices()
        ok = True
        for p in range(n):
            for q in range(n):
                a, b = eq.energies(p, q), oeq.energies_of(p, q)
                if (a is None) != (b is None) or (a is not None and sorted(int(x) for x in a.array.reshape(-1)) !=
                                                  sorted(int(x) for x in np.asarray(b).reshape(-1))):
                    ok = False
        for name in names:
            r, o = eq.relation(geq.std_equivalences.get(name)), oeq.relation(geq.std_equivalences._T[name])
            ok = ok and r.count_classes() == o.count_classes()
        if not ok:
            bad.append(int(seeds[k]))
    out.update({"cpu_baseline": {"value": len(systems) / odt, "unit": UNIT, "cores": 1, "kind": "port",
                                 "sample": f"the same {len(systems)} LTSs, oracle equivalences(), 1 thread"},
                "parity_checked": len(systems), "parity_mismatches": len(bad), "mismatched_seeds": bad[:16]})
    return out


def run_large(ctx, n_states: int, check: bool, pairs: int = 48) -> dict:
    """The large configuration's generator (power-law out-degree, 12 labels,
    tau p 0.15, a strongly connected core of 10 %, 4 transitions per state)
    at n_states states: TransitionSystem::equivalences() of the whole system
    (minimisation, the compare_all game built and solved on the device).  With
    `check` the energies of a sample of start pairs are compared with the
    oracle's TransitionSystem::compare of the same pairs (the energies of a
    position depend only on the part of the game it reaches)."""
    import gpuequiv_b200 as geq
    synth = synth_mod()
    src, dst, lab = synth.large_lts(1, n=n_states, m=4 * n_states)
    lts = geq.TransitionSystem.from_arrays(src, dst, lab)
    times = []
    for _ in range(2):
        t = time.perf_counter()
        eq = lts.equivalences(ctx)
        times.append(time.perf_counter() - t)
    out = {"workload": f"large generator at {n_states} states, {4 * n_states} transitions, 12 labels, tau p 0.15, "
                       f"10 % strongly connected core: equivalences() of the whole system",
           "seconds": min(times), "start_positions": eq.n_starting_points()}
    if not check:
        return out
    from oracle import ora
    rng = np.random.default_rng(5)
    red, mp = ora.Lts.from_arrays(src, dst, lab).bisimilar_minimize()  # as compare() does, once
    gred, gmp = lts.bisimilar_minimize()
    checked = bad = 0
    t_end = time.perf_counter() + 60.0
    for _ in range(pairs * 50):
        if checked >= pairs or time.perf_counter() > t_end:
            break
        p, q = (int(x) for x in rng.integers(0, n_states, 2))
        mine = eq.energies(p, q)
        if p == q or mine is None or mp[p] == mp[q]:
            continue
        # pairs whose own game has at most 20,000 positions (the oracle is
        # sequential): the library's host GameBuild with that bound decides
        try:
            geq.GameBuild.compare_bounded(gred, int(gmp[p]), int(gmp[q]), 20_000)
        except geq.GeqError:
            continue
        b = ora.Build.compare(red, int(mp[p]), int(mp[q]), positions=False)
        ref = ora.run_game(6, 3, b.row, b.col, b.wt, b.attacker, ora.standard_reach(b.row, b.attacker)).lists()[0]
        checked += 1
        if sorted(int(x) for x in mine.array.reshape(-1)) != sorted(int(x) for x in np.asarray(ref).reshape(-1)):
            bad += 1
    out.update({"parity_checked": checked, "parity_mismatches": bad,
                "what": "start-pair energies against the oracle's compare(p, q), pairs whose game has at most "
                        "20,000 positions, at most 60 s of checks"})
    return out


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
    """The reference's path on the host cores: the oracle (the reference's
    Rust/wgpu code cannot run here) builds every job's game with its own
    GameBuild and solves it with its EnergyGame::run on all host threads,
    the threads sharing one work counter, largest games first.  A step is one
    solve of the whole batch -- or, when K steps of it would not end within a
    few minutes, of every s-th job (a sample with the batch's size mix)."""
    if d.rank != 0:
        return
    seeds, rows = batched_seeds(args.jobs, 0)
    threads = os.cpu_count() or 1
    t = time.perf_counter()
    games = build_games_oracle_parallel(seeds, threads)
    build_s = time.perf_counter() - t
    # warm-up: one solve of the whole batch (it also sizes the steps), the
    # others on a small sample
    _, full_s, _ = oracle_solve(games, threads)
    for _ in range(max(0, args.warmup - 1)):
        oracle_solve(games[::64], threads)
    stride = 1
    while stride < 64 and args.steps * full_s / stride > 150.0:
        stride *= 2
    step_games = games[::stride]
    rates = []
    for _ in range(args.steps):
        r, dt, _ = oracle_solve(step_games, threads)
        rates.append((r, dt))
    value = float(np.median([r[0] for r in rates]))
    sample = (f"{len(step_games)} of the {len(games)} games per step" +
              (f" (every {stride}th job)" if stride > 1 else " (the whole batch)") +
              f", oracle GameBuild (untimed, {build_s:.1f} s) + EnergyGame::run on {threads} threads, "
              f"one shared work counter, largest games first")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.median([r[1] for r in rates]) * 1e3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": workload_config(rows, d.world),
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

    progress("resident solve")
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
    clocks = Clocks(d.local_rank)
    clocks.start()
    d.barrier()
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
    # the lists of the last timed solve: checked against the oracle below,
    # and the byte floor of the solve from them
    res_offs, res_data = dg.download_raw()
    b_min = sum(geq.b_min(g, o) for g, o in zip(graphs, res_offs))

    progress("roofline")
    # ---- roofline of the round kernel (one profiled solve, not timed) ----
    ctx.set_tuning(flags=TUNE_PROFILE)
    st_prof = dg.solve()
    ctx.set_tuning(flags=0)
    dg.close()
    peak, peak_kind = peak_hbm()
    k_ms = st_prof["round_kernel_ms"]
    k_launch = max(1, st_prof["round_kernel_launches"])
    achieved = st_prof["algorithmic_bytes"] / (k_ms / 1e3) / 1e9 if k_ms > 0 else None
    alg_per_launch = st_prof["algorithmic_bytes"] / k_launch
    traffic = DRAM_PER_ALGORITHMIC_BYTE * alg_per_launch

    progress("e2e")
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

    progress("lts pipeline")
    # ---- LTS -> verdict: compare_batch from the unminimised LTSs (host
    # minimisation, games built on the device, solved, start energies back) ----
    lts_jobs, lts_pipe = run_lts_pipeline(ctx, seeds, graphs, args, d)

    progress("plain")
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

    progress("serving")
    # ---- serving loop (not part of value) ----
    # game requests drawn from this batch: Poisson arrivals, then saturation
    rates = [float(x) for x in args.serve_rates.split(",") if x.strip()]
    serving = None
    if rates or args.saturation_seconds > 0:
        serving = run_serving(ctx, views, False, rates, args.serve_seconds, 100 + 1000 * d.rank,
                              args.saturation_seconds, n_pipelines=args.serve_pipelines)
        sat = serving["saturation"]
        serving["saturation_vs_plain"] = sat["throughput_games_s"] / plain_rate if sat and plain_rate else None
    # the serving configuration: equivalence queries on LTSs of 20-20,000
    # states (minimised, built and solved on the device), games above the
    # position bound refused
    qrates = [float(x) for x in args.query_rates.split(",") if x.strip()]
    serving_q = None
    if qrates or args.saturation_seconds > 0:
        pool = serving_queries(args.query_pool, seed=7 + 1000 * d.rank)
        # the queries whose game is within the bound (host GameBuild with the
        # bound, on the first 256 of the pool): the saturation run and the
        # plain form both take these, so that they compare like with like
        acc_idx = [i for i in range(min(256, len(pool))) if within_bound(pool[i], args.query_bound)]
        progress("serving: queries")
        serving_q = run_serving(ctx, pool, True, qrates, args.serve_seconds, 200 + 1000 * d.rank,
                                args.saturation_seconds, max_game_positions=args.query_bound,
                                outstanding=256, saturation_items=acc_idx, n_pipelines=args.serve_pipelines)
        # the plain form on the same queries: one compare() call each
        acc = [pool[i] for i in acc_idx[:64]]
        for j in acc[:8]:
            geq.compare_batch([j], context=ctx)
        t = time.perf_counter()
        for j in acc:
            geq.compare_batch([j], context=ctx)
        plain_q = len(acc) / (time.perf_counter() - t) if acc else None
        serving_q["plain_per_query"] = {"value": plain_q, "unit": UNIT,
                                        "sample": f"{len(acc)} pool queries within the bound, one compare() each"}
        serving_q["saturation_queries"] = f"the {len(acc_idx)} of the first 256 pool queries within the bound"
        sat = serving_q["saturation"]
        serving_q["saturation_vs_plain"] = (sat["throughput_games_s"] / plain_q) if sat and plain_q else None

    progress("small")
    # ---- small configuration: equivalences() of 100 seeded 40-state LTSs ----
    small = run_small(ctx, list(range(100)), check=d.rank == 0)
    progress("large")
    large = run_large(ctx, args.large_states, check=d.rank == 0) if args.large_states else None

    progress("stress")
    # ---- stress configuration: one 2M-position / 10M-edge game, resident ----
    stress = None
    if args.stress:
        srow, scol, swt, satt = synth_mod().stress_game()
        sg = geq.GameGraph.from_csr(srow, scol, swt, satt, geq.EnergyConf.STANDARD)
        sdg = geq.DeviceGames([sg], ctx)
        for _ in range(2):
            sdg.solve()
        sts = [sdg.solve() for _ in range(3)]
        s_offs, _ = sdg.download_raw()
        s_bmin = geq.b_min(sg, s_offs[0])
        del s_offs
        flags0 = ctx.tuning()["flags"]
        ctx.set_tuning(flags=flags0 | TUNE_PROFILE)
        s_prof = sdg.solve()
        ctx.set_tuning(flags=flags0)
        sdg.close()
        sms = float(np.median([x["device_ms"] for x in sts]))
        s_ach = s_prof["algorithmic_bytes"] / (s_prof["round_kernel_ms"] / 1e3) / 1e9 if s_prof["round_kernel_ms"] else None
        stress = {"workload": "stress: 2,000,000 positions (60 % attackers), 10,000,000 edges, seed 2, standard reach",
                  "solve_ms": sms, "edges_relaxed": sts[0]["edges_relaxed"],
                  "positions_computed": sts[0]["positions_computed"], "rounds": sts[0]["rounds"],
                  "edges_relaxed_per_s": sts[0]["edges_relaxed"] / (sms / 1e3),
                  "roofline": {"bound": "hbm", "achieved": s_ach, "peak": peak, "unit": "GB/s",
                               "frac": s_ach / peak if s_ach else None, "peak_kind": peak_kind,
                               "kernel": "k_round + k_round_big (all rounds of one solve)",
                               "algorithmic_bytes_per_solve": s_prof["algorithmic_bytes"],
                               "round_kernel_ms_per_solve": s_prof["round_kernel_ms"],
                               "round_kernel_launches": s_prof["round_kernel_launches"],
                               "b_min": s_bmin, "b_min_over_algorithmic_bytes": s_bmin / s_prof["algorithmic_bytes"]}}

    progress("cpu baseline")
    # ---- CPU baseline: the oracle on one host thread (rank 0, N=1), on every
    # 16th job; its lists are the check of the timed solve's lists ----
    cpu, parity = None, None
    if d.rank == 0:
        cidx = sample_indices(len(seeds), 256)
        cg = build_games_oracle_parallel([seeds[i] for i in cidx], os.cpu_count() or 4)
        threads = 1 if d.world == 1 else (os.cpu_count() or 4)
        r, dt, sols = oracle_solve(cg, threads)
        if d.world == 1:
            cpu = {"value": r, "unit": UNIT, "cores": 1, "kind": "port",
                   "sample": f"{len(cg)} games (every {max(1, len(seeds) // 256)}th job of the batch) in {dt:.1f} s, "
                             f"oracle EnergyGame::run, 1 thread"}
        bad = []
        for i, sol in zip(cidx, sols):
            same = (len(res_offs[i]) == len(sol.offsets) and
                    all(np.array_equal(a, b) for a, b in zip(canonical(res_offs[i], res_data[i]),
                                                             canonical(sol.offsets, sol.data))))
            if not same:
                bad.append(int(i))
        parity = {"parity_checked": len(cidx), "parity_mismatches": len(bad), "mismatched_jobs": bad[:16],
                  "what": "every position's list (as a set) of the last timed solve against the oracle's "
                          "GameBuild + EnergyGame::run, every 16th job"}
    del res_offs, res_data

    if d.rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": d.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": workload_config(rows, d.world),
            "host_build_s": round(build_s, 2),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "traffic_source": f"ncu DRAM bytes per algorithmic byte ({DRAM_PER_ALGORITHMIC_BYTE}) of all "
                                           "round-kernel launches (k_round + k_round_big) of the 1024-job case x "
                                           "algorithmic bytes per full-size round",
                         "b_min": b_min, "b_min_over_algorithmic_bytes": b_min / st_prof["algorithmic_bytes"],
                         "b_min_note": "schedule-independent floor 4(n+1) + 8m + n + sum_v 4|A*_v|(1+indeg v) "
                                       "from the final lists",
                         "algorithmic_bytes_per_launch": alg_per_launch,
                         "kernel": "k_round + k_round_big (one round)", "peak_kind": peak_kind,
                         "algorithmic_bytes_per_solve": st_prof["algorithmic_bytes"],
                         "round_kernel_ms_per_solve": k_ms, "round_kernel_launches": k_launch},
            "cpu_baseline": cpu,
            **(parity or {}),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(in_bytes),
                    "d2h_bytes_per_step": int(out_bytes)},
            "plain_cuda": {"value": plain_rate, "unit": UNIT, "sample": f"{len(idx)} games (every "
                           f"{max(1, len(graphs) // len(idx))}th job), one geq_energy_game_run call each"},
            "batched_vs_plain": value / plain_rate if plain_rate else None,
            "lts_pipeline": lts_pipe,
            "small": small,
            "large_single": large,
            "stress": stress,
            "serving": {"workload": "game requests (geq_server_submit) drawn from this batch's games: Poisson "
                                    "arrivals, then a closed loop of 8192 requests in flight (saturation); "
                                    f"geq_server with {args.serve_pipelines or 3} pipelines, 150 GB admission "
                                    "budget; load from native threads; latency = submit -> lists in the "
                                    "caller's hands",
                        **(serving or {}),
                        "queries": {"workload": f"serving configuration: Poisson arrivals of compare(p, q) queries "
                                                f"on seeded LTSs of log-uniform 20-20,000 states (pool of "
                                                f"{args.query_pool}), geq_server_submit_compare (minimisation, "
                                                f"GameBuild, solve on the device), games above "
                                                f"{args.query_bound} positions refused; then a closed loop of 256 "
                                                f"queries in flight", **(serving_q or {})}},
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
    if parity and parity["parity_mismatches"]:
        raise SystemExit(f"parity: {parity['parity_mismatches']} of {parity['parity_checked']} checked jobs differ "
                         f"from the oracle: {parity['mismatched_jobs']}")
    if large and large.get("parity_mismatches"):
        raise SystemExit(f"parity: large single LTS, {large['parity_mismatches']} start pairs differ from the oracle")
    if small and small.get("parity_mismatches"):
        raise SystemExit(f"parity: small configuration, seeds {small['mismatched_seeds']} differ from the oracle")


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
