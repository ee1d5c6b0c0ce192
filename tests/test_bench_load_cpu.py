"""bench.py's serving load driver (the native driver of
gpuequiv_b200/csrc/loadgen.cpp behind bench.Load) against a fake server on
the CPU: every submitted request is collected once from the completion
queue, with its own latency, in open and closed loop, also when requests
finish out of order or not before the drain deadline."""
import ctypes as C
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


class FakeServer:
    """submit / poll_any / free as C callbacks: request k finishes delay(k)
    seconds after its submission, in whatever order that gives; every 7th
    answers with status 2."""

    def __init__(self, delay):
        self.delay = delay
        self.mu = threading.Lock()
        self.next = 1
        self.pending = []  # (finish time, ticket)
        self.freed = 0
        self.inflight = 0
        self.max_seen = 0
        self.cb = (bench.LoadApi.SUBMIT(self.submit), bench.LoadApi.POLL(self.poll_any), bench.LoadApi.FREE(self.free))
        bench._loadgen()  # the structures' fields
        self.api = bench.LoadApi.Api(None, *self.cb)

    def submit(self, ctx, item, t):
        with self.mu:
            k = self.next
            self.next += 1
            self.pending.append((time.perf_counter() + self.delay(k), k))
            self.inflight += 1
            self.max_seen = max(self.max_seen, self.inflight)
        t[0] = k
        return 0

    def poll_any(self, ctx, timeout_ms, t, sol):
        end = time.perf_counter() + timeout_ms / 1e3
        while True:
            with self.mu:
                now = time.perf_counter()
                ready = [x for x in self.pending if x[0] <= now]
                if ready:
                    x = min(ready)
                    self.pending.remove(x)
                    self.inflight -= 1
                    t[0] = x[1]
                    if x[1] % 7 == 0:
                        return 2
                    sol[0] = 1
                    return 0
            if time.perf_counter() > end:
                t[0] = 0
                return 4
            time.sleep(0.0002)

    def free(self, sol):
        with self.mu:
            self.freed += 1


def make_load(fake, drain_s=10.0):
    return bench.Load(None, None, False, threads=4, drain_s=drain_s, api=fake.api)


def test_unfinished_requests_count_at_the_deadline():
    fake = FakeServer(lambda k: 30.0 if k == 3 else 0.001)  # request 3 never finishes in time
    lat, status, span = make_load(fake, drain_s=0.3).open_loop(np.linspace(0, 0.05, 20), np.zeros(20, np.int64))
    assert len(status) == 20 and (status == -1).sum() == 1 and (status >= 0).sum() == 19
    assert span < 5


def test_open_loop_collects_every_request_once():
    fake = FakeServer(lambda k: 0.02 if k % 5 == 0 else 0.001)  # every 5th finishes late
    n = 400
    lat, status, span = make_load(fake).open_loop(np.linspace(0, 0.2, n), np.zeros(n, np.int64))
    assert len(lat) == n and len(status) == n and (status >= 0).all()
    assert (status == 2).sum() == len([k for k in range(1, n + 1) if k % 7 == 0])
    assert fake.freed == (status == 0).sum()
    assert np.percentile(lat, 50) < 10 and lat.max() >= 19  # the late ones do not hold back the others
    assert 0.2 <= span < 2.0


def test_closed_loop_keeps_outstanding_bounded():
    fake = FakeServer(lambda k: 0.002)
    lat, status, span = make_load(fake).closed_loop(np.zeros(4, np.int64), 16, 0.3)
    assert len(lat) == len(status) > 50 and (status >= 0).all()
    assert fake.max_seen <= 16
    assert lat.max() < 1000


def test_refused_submits_are_recorded_at_once():
    """A submit that fails (a full queue, a malformed game) is recorded with
    its status and never waited for."""
    fake = FakeServer(lambda k: 0.001)
    real_submit = fake.submit

    def submit(ctx, item, t):
        if item == 1:
            t[0] = 0
            return 7  # GEQ_ERR_BUSY
        return real_submit(ctx, item, t)

    fake.cb = (bench.LoadApi.SUBMIT(submit),) + fake.cb[1:]
    fake.api = bench.LoadApi.Api(None, *fake.cb)
    pick = np.array([0, 1] * 50, np.int64)
    lat, status, span = make_load(fake, drain_s=2.0).open_loop(np.linspace(0, 0.05, 100), pick)
    assert (status[pick == 1] == 7).all()
    assert (status[pick == 0] >= 0).all() and (status[pick == 0] != 7).all()
    assert span < 3
