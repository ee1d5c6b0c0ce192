"""The multi-rank path of bench.py on CPU: two gloo ranks.

Under torchrun every rank solves its own batch (weak scaling, replicas, no
collective on the data path); the only collectives are the barrier and the
max / sum of the timings.  This test runs that host logic with world size 2
on the CPU: rank 0 takes the committed manifest's jobs, rank 1 draws its own
seeds from a disjoint range, and the reductions give the max and the sum over
ranks.
"""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

RANK_SCRIPT = r"""
import json, os, sys
sys.path.insert(0, os.environ["GEQ_ROOT"])
import bench
d = bench.Dist(backend="gloo")
seeds, rows = bench.batched_seeds(3, d.rank)
d.barrier()
out = {"rank": d.rank, "world": d.world, "seeds": seeds, "sizes": [r[1] for r in rows],
       "max": d.max(float(10 + d.rank)), "sum": d.sum(float(len(seeds)))}
d.close()
print("RESULT " + json.dumps(out), flush=True)
"""


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_bench_plumbing(tmp_path):
    script = tmp_path / "rank.py"
    script.write_text(RANK_SCRIPT)
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, GEQ_ROOT=ROOT, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                   LOCAL_RANK=str(rank), WORLD_SIZE="2", CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    results = {}
    for p in procs:
        try:
            out, err = p.communicate(timeout=300)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            pytest.fail("a gloo rank did not finish")
        assert p.returncode == 0, err[-2000:]
        line = [l for l in out.splitlines() if l.startswith("RESULT ")][-1]
        r = json.loads(line[len("RESULT "):])
        results[r["rank"]] = r
    r0, r1 = results[0], results[1]
    assert r0["world"] == r1["world"] == 2
    # rank 0: the manifest's first jobs; rank 1: its own seed range
    from gpuequiv_b200 import synth
    manifest = synth.batched_manifest()["jobs"][:3]
    assert r0["seeds"] == [row[0] for row in manifest]
    assert r0["sizes"] == [row[1] for row in manifest]
    assert len(r1["seeds"]) == 3 and min(r1["seeds"]) >= 1_000_000
    assert not set(r0["seeds"]) & set(r1["seeds"])
    assert all(0 < n <= 200_000 for n in r1["sizes"])
    # reductions: max of the step times, sum of the games
    assert r0["max"] == r1["max"] == 11.0
    assert r0["sum"] == r1["sum"] == 6.0
