"""The batched sweep's host logic on the CPU (mom25d_b200.batch): a sweep is a set of requests present at the
start, all of them served by the slots at once, each result returned in frequency order; |dS| is the largest
entry difference over the frequencies compared. The solve is a stand-in."""
import threading
import time

import numpy as np

from mom25d_b200.batch import batched_sweep, max_dS, sweep_requests
from mom25d_b200.serve import GB, Server


def test_sweep_runs_every_frequency_concurrently_in_order():
    lock = threading.Lock()
    seen = {'now': 0, 'max': 0}

    def solve(slot, key, f):
        with lock:
            seen['now'] += 1
            seen['max'] = max(seen['max'], seen['now'])
        time.sleep(0.02)
        with lock:
            seen['now'] -= 1
        return np.array([[f, slot]], complex), dict(path='fresh', iters=[3])

    freqs = np.linspace(1e9, 6e9, 12)
    srv = Server({'b': None}, slots=4, budget_bytes=100 * GB, solve=solve, sizes={'b': 8000}, ports={'b': 2},
                 resident=lambda slot, key: 0.0, evict=lambda slot, key: None)
    S, wall, reqs = batched_sweep(srv, 'b', freqs, multi=False)
    assert [s[0, 0].real for s in S] == list(freqs)          # frequency order, whatever the completion order
    assert seen['max'] == 4 and all(r.path == 'fresh' for r in reqs)
    assert wall < 12 * 0.02                                   # overlapped, not one after another
    assert [r.f for r in sweep_requests('b', freqs)] == list(freqs)


def test_max_dS():
    A = [np.eye(2), np.zeros((2, 2))]
    B = [np.eye(2) + 1e-6, np.full((2, 2), 3e-5j)]
    assert abs(max_dS(A, B) - 3e-5) < 1e-12
