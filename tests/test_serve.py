"""The serving loop's host logic on the CPU (mom25d_b200.serve): continuous admission by slots and device-memory
footprint, with the idle solvers' resident state counted and evicted least recently used first when a request
would not fit; first come first served; every request completed with its own result and latency. The solve is a
stand-in that records the concurrency and the bytes it sees."""
import threading
import time

import numpy as np

from mom25d_b200.serve import GB, Request, Server, footprint_bytes, poisson_requests, resident_estimate


class FakeSolve:
    """Stands in for the GPU solve: sleeps in proportion to the board's size, records the requests in flight, and
    keeps the resident state of each (slot, board) solver it has made (half the estimate) until evicted."""

    def __init__(self, srv_sizes, budget):
        self.lock = threading.Lock()
        self.in_flight, self.bytes, self.max_in_flight, self.max_bytes = 0, 0.0, 0, 0.0
        self.sizes, self.budget = srv_sizes, budget
        self.order, self.solvers, self.evicted = [], {}, []

    def resident(self, slot, key):
        return self.solvers.get((slot, key), 0.0)

    def evict(self, slot, key):
        with self.lock:
            self.evicted.append((slot, key))
            self.solvers.pop((slot, key), None)

    def __call__(self, slot, key, f):
        fp = footprint_bytes(self.sizes[key], 2)
        with self.lock:
            new = (slot, key) not in self.solvers
            self.solvers.setdefault((slot, key), 0.5 * resident_estimate(self.sizes[key]))
            self.in_flight += 1
            self.bytes += fp
            self.max_in_flight = max(self.max_in_flight, self.in_flight)
            held = self.bytes + sum(self.solvers.values())
            self.max_bytes = max(self.max_bytes, held)
            self.order.append((key, f))
        time.sleep(0.01 + 0.002 * (self.sizes[key] / 1000.0))
        S = np.array([[f / 1e9, len(key)], [self.sizes[key], slot * 0 + 1.0]], complex)
        with self.lock:
            self.in_flight -= 1
            self.bytes -= fp
        return S, dict(path='fake', iters=[1])


def _server(sizes, budget, slots, fake):
    return Server({k: None for k in sizes}, slots=slots, budget_bytes=budget, solve=fake, sizes=sizes,
                  ports={k: 2 for k in sizes}, resident=fake.resident, evict=fake.evict)


def test_footprint_is_the_librarys_workspace_and_the_matrices():
    from mom25d_b200 import _lib
    import ctypes
    L = _lib.lib()
    n = 18788
    fp = footprint_bytes(n, 8)
    ws = L.m25_getrf_workspace(ctypes.c_int(n), ctypes.c_int(1)) + L.m25_getrs_aux_bytes(ctypes.c_int(n), ctypes.c_int(1))
    assert 24.0 * n * n + ws < fp < 24.0 * n * n + ws + 0.2 * GB


def test_admission_by_slots_and_footprint():
    sizes = {'small': 2000, 'big': 20000}
    budget = footprint_bytes(20000, 2) + footprint_bytes(2000, 2) + resident_estimate(20000) + \
        3 * resident_estimate(2000) + 0.2 * GB
    fake = FakeSolve(sizes, budget)
    srv = _server(sizes, budget, 3, fake)
    reqs = [Request(i, 'big' if i % 3 == 0 else 'small', 1e9 + i * 1e8, 0.002 * i) for i in range(12)]
    t = time.perf_counter()
    out = srv.run(reqs)
    wall = time.perf_counter() - t
    assert all(r.error is None and r.S is not None for r in out)
    assert fake.max_in_flight <= 3
    assert fake.max_bytes <= budget and srv.peak_bytes <= budget      # in flight + resident, never above the budget
    for r in out:                                         # each request's own result, whatever ran beside it
        assert r.S[0, 0] == r.f / 1e9 and r.S[1, 0] == sizes[r.board]
        assert r.latency >= 0 and r.done >= r.start >= r.arrival - 1e-3
    rep = Server.report(out, wall)
    assert rep['requests'] == 12 and rep['errors'] == 0 and rep['p99_ms'] >= rep['p50_ms']


def test_idle_solvers_are_evicted_to_make_room():
    sizes = {'a': 10000, 'b': 10000, 'c': 10000}
    budget = footprint_bytes(10000, 2) + 1.5 * resident_estimate(10000) + 0.1 * GB   # one board's solver at a time
    fake = FakeSolve(sizes, budget)
    srv = _server(sizes, budget, 1, fake)
    reqs = [Request(i, 'abc'[i % 3], 1e9, 0.001 * i) for i in range(6)]
    out = srv.run(reqs)
    assert all(r.error is None for r in out)
    assert len(fake.evicted) >= 2 and srv.peak_bytes <= budget and fake.max_bytes <= budget
    assert (0, 'c') in srv.resident and len(srv.resident) <= 2         # the last board's solver stays resident


def test_first_come_first_served_and_oversize_rejected():
    sizes = {'a': 1000}
    fake = FakeSolve(sizes, 1e12)
    srv = _server(sizes, 1e12, 1, fake)
    reqs = [Request(i, 'a', (5 - i) * 1e9, 0.001 * i) for i in range(5)]
    srv.run(reqs)
    assert [f for _, f in fake.order] == [r.f for r in sorted(reqs, key=lambda r: r.arrival)]
    small = _server(sizes, 1.0, 1, fake)
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
