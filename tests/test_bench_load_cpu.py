"""bench.py's serving load driver (Load) against a fake server on the CPU:
every submitted request is collected once from the completion queue, with
its own latency, in open and closed loop, also when requests finish out of
order."""
import ctypes as C
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


class FakeLib:
    """geq_server_submit / _poll_any / geq_solution_free: request k finishes
    delay(k) seconds after its submission, in whatever order that gives."""

    def __init__(self, delay):
        self.delay = delay
        self.mu = threading.Lock()
        self.next = 1
        self.pending = []  # (finish time, ticket)
        self.freed = 0

    def geq_server_submit(self, h, item, t):
        with self.mu:
            k = self.next
            self.next += 1
            self.pending.append((time.perf_counter() + self.delay(k), k))
        C.cast(t, C.POINTER(C.c_uint64)).contents.value = k
        return 0

    def geq_server_poll_any(self, h, timeout_ms, t, sol):
        end = time.perf_counter() + timeout_ms / 1e3
        while True:
            with self.mu:
                now = time.perf_counter()
                ready = [x for x in self.pending if x[0] <= now]
                if ready:
                    x = min(ready)
                    self.pending.remove(x)
                    C.cast(t, C.POINTER(C.c_uint64)).contents.value = x[1]
                    return 2 if x[1] % 7 == 0 else 0
            if time.perf_counter() > end:
                return 4
            time.sleep(0.0002)

    def geq_solution_free(self, sol):
        self.freed += 1


def make_load(delay):
    load = bench.Load.__new__(bench.Load)
    load.lib, load.h, load.items, load.queries, load.threads = FakeLib(delay), None, [C.c_int(0)] * 4, False, 4
    load.drain_s = 10.0
    return load


def test_unfinished_requests_count_at_the_deadline():
    load = make_load(lambda k: 30.0 if k == 3 else 0.001)  # request 3 never finishes in time
    load.drain_s = 0.3
    lat, status, span = load.open_loop(np.linspace(0, 0.05, 20), np.zeros(20, np.int64))
    assert len(status) == 20 and (status == -1).sum() == 1 and len(lat) == 19
    assert span < 5


def test_open_loop_collects_every_request_once():
    load = make_load(lambda k: 0.02 if k % 5 == 0 else 0.001)  # every 5th finishes late
    n = 400
    lat, status, span = load.open_loop(np.linspace(0, 0.2, n), np.zeros(n, np.int64))
    assert len(lat) == n and len(status) == n
    assert (status == 2).sum() == len([k for k in range(1, n + 1) if k % 7 == 0])
    assert np.percentile(lat, 50) < 10 and lat.max() >= 19  # the late ones do not hold back the others
    assert 0.2 <= span < 2.0


def test_closed_loop_keeps_outstanding_bounded():
    load = make_load(lambda k: 0.002)
    lat, status, span = load.closed_loop(np.zeros(4, np.int64), 16, 0.3)
    assert len(lat) == len(status) > 50
    assert lat.max() < 1000
