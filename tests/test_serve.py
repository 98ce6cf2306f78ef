"""The serving loop's host logic on the CPU (mom25d_b200.serve): continuous admission by slots and device-memory
footprint, first come first served, every request completed with its own result and latency. The solve is a
stand-in that records the concurrency it sees."""
import threading
import time

import numpy as np

from mom25d_b200.serve import GB, Request, Server, footprint_bytes, poisson_requests


class FakeSolve:
    def __init__(self, srv_sizes, budget):
        self.lock = threading.Lock()
        self.in_flight, self.bytes, self.max_in_flight, self.max_bytes = 0, 0.0, 0, 0.0
        self.sizes, self.budget = srv_sizes, budget
        self.order = []

    def __call__(self, slot, key, f):
        fp = footprint_bytes(self.sizes[key])
        with self.lock:
            self.in_flight += 1
            self.bytes += fp
            self.max_in_flight = max(self.max_in_flight, self.in_flight)
            self.max_bytes = max(self.max_bytes, self.bytes)
            self.order.append((key, f))
        time.sleep(0.01 + 0.002 * (self.sizes[key] / 1000.0))
        S = np.array([[f / 1e9, len(key)], [self.sizes[key], slot * 0 + 1.0]], complex)
        with self.lock:
            self.in_flight -= 1
            self.bytes -= fp
        return S, dict(path='fake', iters=[1])


def test_admission_by_slots_and_footprint():
    sizes = {'small': 2000, 'big': 20000}
    budget = footprint_bytes(20000) + footprint_bytes(2000) + 0.5 * GB   # one big and one small at a time
    fake = FakeSolve(sizes, budget)
    srv = Server({'small': None, 'big': None}, slots=3, budget_bytes=budget, solve=fake, sizes=sizes)
    reqs = [Request(i, 'big' if i % 3 == 0 else 'small', 1e9 + i * 1e8, 0.002 * i) for i in range(12)]
    t = time.perf_counter()
    out = srv.run(reqs)
    wall = time.perf_counter() - t
    assert all(r.error is None and r.S is not None for r in out)
    assert fake.max_in_flight <= 3
    assert fake.max_bytes <= budget
    for r in out:                                         # each request's own result, whatever ran beside it
        assert r.S[0, 0] == r.f / 1e9 and r.S[1, 0] == sizes[r.board]
        assert r.latency >= 0 and r.done >= r.start >= r.arrival - 1e-3
    rep = Server.report(out, wall)
    assert rep['requests'] == 12 and rep['errors'] == 0 and rep['p99_ms'] >= rep['p50_ms']


def test_first_come_first_served_and_oversize_rejected():
    sizes = {'a': 1000}
    fake = FakeSolve(sizes, 1e12)
    srv = Server({'a': None}, slots=1, budget_bytes=1e12, solve=fake, sizes=sizes)
    reqs = [Request(i, 'a', (5 - i) * 1e9, 0.001 * i) for i in range(5)]
    srv.run(reqs)
    assert [f for _, f in fake.order] == [r.f for r in sorted(reqs, key=lambda r: r.arrival)]
    small = Server({'a': None}, slots=1, budget_bytes=1.0, solve=fake, sizes=sizes)
    try:
        small.run([Request(0, 'a', 1e9)])
        assert False, 'a request above the budget must be refused'
    except MemoryError:
        pass


def test_poisson_requests_are_seeded():
    a = poisson_requests(['x', 'y'], [0.7, 0.3], 20.0, 50, seed=3)
    b = poisson_requests(['x', 'y'], [0.7, 0.3], 20.0, 50, seed=3)
    assert [(r.board, r.f, r.arrival) for r in a] == [(r.board, r.f, r.arrival) for r in b]
    assert all(0.5e9 <= r.f <= 10e9 for r in a) and np.all(np.diff([r.arrival for r in a]) > 0)
