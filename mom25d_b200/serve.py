"""
mom25d_b200.serve - (board, frequency) solves served as they arrive, several at once on one GPU.

    python -m mom25d_b200.serve [--rate 20] [--requests 40] [--slots 4] [--seed 0]

The serving mode of the hot path (the reference solves one board's sweep at a time, sim.py:331 /
run.py:41; this is the request loop a service puts in front of it):

  - boards stay resident: each board's mesh, near-pair lists and device geometry are built on its first request
    and kept, one solver per (board, slot), so later requests for the board pay only the per-frequency work;
  - continuous batching: a request is admitted as soon as it has arrived, a slot is free and its device-memory
    footprint (footprint_bytes: the double Z, its complex64 copy, the library's LU and solve workspaces and the
    Krylov bases) fits the budget beside the requests in flight and the resident state of every board solver
    (mesh, near pairs and their kept moments: counted until the solver is evicted); admitted requests run
    concurrently, each slot on its own CUDA stream and host thread (the library's calls release the interpreter
    lock), so their kernels overlap on the device;
  - a finished request gives its per-frequency buffers back (DirectSolver.release), so an idle solver holds only
    its resident state; where a request would not fit, idle solvers are evicted least recently used first;
  - results do not depend on the mix: no reduction crosses requests and kept-LU reuse is off here (a reused
    factor would make a request's iterations depend on the one before it), so a request's S is the same alone and
    in the mix up to the rounding of the near field's atomic additions;
  - latency is completion minus arrival; p50 / p99 and solves / s are reported.

Request.S holds the scattering matrix (nports x nports complex).
"""
import argparse
import heapq
import json
import queue
import threading
import time

import numpy as np

GB = 1e9


class Request:
    __slots__ = ('rid', 'board', 'f', 'arrival', 'start', 'done', 'S', 'error', 'slot', 'path', 'iters', 'far')

    def __init__(self, rid, board, f, arrival=0.0, far=None):
        self.rid, self.board, self.f, self.arrival = rid, board, float(f), float(arrival)
        self.far = far                  # Z with the far part at f already filled (the batched sweep), a callable
                                        # returning it when ready, or None
        self.start = self.done = None
        self.S = self.error = self.slot = self.path = None
        self.iters = []

    @property
    def latency(self):
        return None if self.done is None else self.done - self.arrival


RESTART = 30                   # the refinement's Krylov depth (operator.MIXED_MAX_ITER)


def footprint_bytes(N, ports=8):
    """Device memory one mixed-precision request holds while it runs (operator.DirectSolver._solve_kept): the double
    Z (16 N^2) and its complex64 copy factored in place (8 N^2); the LU workspace (m25_getrf_workspace) and the
    solve data of the factor (m25_getrs_aux_bytes), as the library sizes them; the Krylov bases, V (restart + 1
    blocks) and the preconditioned directions (restart blocks) of N x ports complex128; a dozen N x ports vectors
    and the per-frequency tables (16 MB)."""
    import ctypes
    from ._lib import lib
    L = lib()
    ws = int(L.m25_getrf_workspace(ctypes.c_int(int(N)), ctypes.c_int(1)))
    aux = int(L.m25_getrs_aux_bytes(ctypes.c_int(int(N)), ctypes.c_int(1)))
    krylov = (2 * RESTART + 1) * N * ports * 16
    return 24.0 * N * N + ws + aux + krylov + 12 * N * ports * 16 + 16e6


def resident_estimate(N):
    """Device bytes of a board solver's resident state before it exists: about 200 near pairs an unknown, each with
    its two triangle indices and 12 kept analytic moments (104 bytes), plus the mesh arrays (~1 KB an unknown)."""
    return 200 * N * 104 + 1024 * N


class Server:
    """Serves Request objects for the boards given as {key: Board}. solve(slot, key, f) -> (S, info) can be
    replaced (tests drive the admission logic with a stand-in on the CPU); the default solves on the GPU.
    resident(slot, key) -> bytes: a board solver's resident device state (the default measures the solver), and
    evict(slot, key): drops an idle solver."""

    def __init__(self, boards, slots=4, budget_bytes=None, precision='mixed', solve=None, sizes=None, ports=None,
                 resident=None, evict=None):
        self.boards = dict(boards)
        self.slots = int(slots)
        self.precision = precision
        self._sizes = dict(sizes or {})
        self._ports = dict(ports or {})
        self._geo, self._solvers, self._streams = {}, {}, {}
        self._lock = threading.Lock()
        self._solve = solve or self._solve_gpu
        self._resident_of = resident or self._resident_gpu
        self._evict = evict or self._evict_gpu
        self.resident = {}                                # (slot, key) -> bytes held between requests
        self._last_use = {}
        if budget_bytes is None:
            import torch
            free, _ = torch.cuda.mem_get_info()
            budget_bytes = 0.8 * free
        self.budget = float(budget_bytes)
        self.peak_bytes = 0.0                             # the most in-flight + resident bytes admitted at once

    # ---- the per-board state, built on first use -----------------------------------------------------------------
    def size(self, key):
        if key not in self._sizes:
            self._sizes[key] = self._geometry(key).N
        return self._sizes[key]

    def ports(self, key):
        if key not in self._ports:
            self._ports[key] = max(1, len(self._geometry(key).ports))
        return self._ports[key]

    def _geometry(self, key):
        with self._lock:
            if key not in self._geo:
                from .geometry import Geometry
                self._geo[key] = Geometry(self.boards[key])
            return self._geo[key]

    def _solver(self, slot, key):
        import torch
        from .operator import DirectSolver
        from . import umma_available
        if slot not in self._streams:
            self._streams[slot] = torch.cuda.Stream()
        if (slot, key) not in self._solvers:
            with torch.cuda.stream(self._streams[slot]):
                ds = DirectSolver(self._geometry(key), stream=self._streams[slot], tf32=umma_available())
                ds.reuse = False                       # results independent of the request order
                ds.hybrid = True                       # the admission has reserved the double Z's room
                self._solvers[(slot, key)] = ds
        return self._solvers[(slot, key)], self._streams[slot]

    def _solve_gpu(self, slot, key, f, far=None):
        import torch
        from .operator import SolveFailed
        ds, stream = self._solver(slot, key)
        geo = self._geometry(key)
        with torch.cuda.stream(stream):
            try:
                if far is not None:
                    stream.wait_stream(torch.cuda.default_stream())    # (filled and synchronised before)
                try:
                    X = ds.solve_direct(f, geo.excitation(), precision=self.precision, far=far)
                except SolveFailed:                     # (sim.py's rule: the frequency again in double precision)
                    X = ds.solve_direct(f, geo.excitation(), precision='double')
                S = geo.sparams_from_currents(X.cpu().numpy(), f)
                stream.synchronize()
                del X
            finally:
                ds.release()                          # the per-frequency buffers go back; the board state stays
        return S, dict(path=ds.last_path, iters=list(ds.iters))

    def _resident_gpu(self, slot, key):
        ds = self._solvers.get((slot, key))
        return float(ds.resident_bytes()) if ds is not None else 0.0

    def _evict_gpu(self, slot, key):
        self._solvers.pop((slot, key), None)

    def footprint(self, key):
        return footprint_bytes(self.size(key), self.ports(key))

    def _cost(self, slot, key):
        """Bytes a request for `key` on `slot` adds while it runs: its footprint, and the board state of the slot's
        solver for the board where that does not exist yet."""
        extra = 0.0 if (slot, key) in self.resident else resident_estimate(self.size(key))
        return self.footprint(key) + extra

    # ---- the loop ------------------------------------------------------------------------------------------------
    def run(self, requests, clock=time.perf_counter):
        """Serves the requests (arrival times in seconds from the call) and returns them completed."""
        reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        for r in reqs:
            need = self.footprint(r.board) + resident_estimate(self.size(r.board))
            if need > self.budget:
                raise MemoryError(f"request {r.rid}: board {r.board!r} needs {need / GB:.1f} GB, above the serving "
                                  f"budget of {self.budget / GB:.1f} GB")
        t0 = clock()
        done_q = queue.Queue()
        work_qs = [queue.Queue() for _ in range(self.slots)]

        def worker(slot):
            while True:
                r = work_qs[slot].get()
                if r is None:
                    return
                r.start = clock() - t0
                try:
                    far = r.far() if callable(r.far) else r.far        # (a callable: wait for the fill)
                    r.far = None
                    r.S, info = self._solve(slot, r.board, r.f) if far is None else \
                        self._solve(slot, r.board, r.f, far=far)
                    del far
                    r.path, r.iters = info.get('path'), info.get('iters', [])
                except Exception as e:                   # reported on the request; the loop keeps serving
                    r.error = f"{type(e).__name__}: {e}"
                r.done = clock() - t0
                done_q.put((slot, r))

        threads = [threading.Thread(target=worker, args=(s,), daemon=True) for s in range(self.slots)]
        for t in threads:
            t.start()
        free_slots = list(range(self.slots))
        in_flight, flight_bytes = 0, 0.0
        busy = set()                                      # (slot, key) solvers running a request
        cost_of = {}
        waiting = []                                      # arrived, not yet admitted: (arrival, rid, request)
        i = 0

        def held():
            return flight_bytes + sum(self.resident.values())

        def make_room(slot, key, need):
            """Evicts idle solvers, least recently used first, until `need` more bytes fit; True when they do."""
            while held() + need > self.budget:
                idle = [k for k in self.resident if k not in busy and k != (slot, key)]
                if not idle:
                    return False
                k = min(idle, key=lambda k: self._last_use.get(k, -1.0))
                self._evict(*k)
                del self.resident[k]
                need = self._cost(slot, key)
            return True

        try:
            while i < len(reqs) or waiting or in_flight:
                now = clock() - t0
                while i < len(reqs) and reqs[i].arrival <= now:
                    heapq.heappush(waiting, (reqs[i].arrival, reqs[i].rid, reqs[i]))
                    i += 1
                # admit in arrival order while a slot is free and the request fits (first come, first served)
                while waiting and free_slots:
                    r = waiting[0][2]
                    slot = free_slots[0]
                    need = self._cost(slot, r.board)
                    if held() + need > self.budget and not make_room(slot, r.board, need):
                        break
                    need = self._cost(slot, r.board)
                    heapq.heappop(waiting)
                    free_slots.pop(0)
                    r.slot = slot
                    cost_of[r.rid] = need
                    flight_bytes += need
                    busy.add((slot, r.board))
                    self.peak_bytes = max(self.peak_bytes, held())
                    in_flight += 1
                    work_qs[slot].put(r)
                if waiting and not in_flight and not free_slots:
                    raise RuntimeError("serving loop: no slot free and nothing in flight")
                if waiting and in_flight == 0 and free_slots:
                    raise MemoryError(f"request {waiting[0][2].rid} does not fit the budget even with every idle "
                                      f"solver evicted")
                timeout = None
                if i < len(reqs):
                    timeout = max(0.0, reqs[i].arrival - (clock() - t0))
                if in_flight == 0 and timeout is not None:
                    time.sleep(timeout)
                    continue
                try:
                    slot, r = done_q.get(timeout=timeout if timeout is not None else 3600.0)
                except queue.Empty:
                    continue
                free_slots.append(slot)
                free_slots.sort()
                flight_bytes -= cost_of.pop(r.rid)
                busy.discard((slot, r.board))
                self.resident[(slot, r.board)] = float(self._resident_of(slot, r.board))
                self._last_use[(slot, r.board)] = clock() - t0
                in_flight -= 1
        finally:
            for q in work_qs:
                q.put(None)
            for t in threads:
                t.join(timeout=60)
        return reqs

    @staticmethod
    def report(reqs, wall):
        lat = np.array([r.latency for r in reqs if r.error is None])
        return dict(requests=len(reqs), errors=sum(r.error is not None for r in reqs),
                    error_messages=sorted({r.error for r in reqs if r.error is not None})[:3],
                    solves_per_s=round(len(lat) / wall, 3) if wall > 0 else None,
                    p50_ms=round(1000 * float(np.percentile(lat, 50)), 1) if len(lat) else None,
                    p99_ms=round(1000 * float(np.percentile(lat, 99)), 1) if len(lat) else None)


def poisson_requests(keys, weights, rate, count, fmin=0.5e9, fmax=10e9, seed=0):
    """Seeded Poisson arrivals at `rate` per second; board drawn with `weights`, frequency U[fmin, fmax]."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, count))
    w = np.asarray(weights, float) / np.sum(weights)
    boards = rng.choice(len(keys), size=count, p=w)
    fs = rng.uniform(fmin, fmax, count)
    return [Request(i, keys[b], fs[i], t[i]) for i, b in enumerate(boards)]


def board_pool(seed=0, targets=(2000, 5000, 10000, 20000, 40000)):
    """Seeded synthetic routed boards of about the given unknown counts: the 20k-unknown generator with the trace
    count and the area scaled by N / 20000 (the unknown count follows the copper area)."""
    from .board import routed_board
    pool = {}
    for j, n in enumerate(targets):
        s = n / 20000.0
        pool[f"routed_{n}"] = routed_board(seed=seed + j, n_traces=max(2, int(round(24 * s))),
                                           n_vias=max(2, int(round(16 * s))), n_ports=max(2, min(8, int(round(8 * s)))),
                                           size=(60e-3 * s ** 0.5, 40e-3 * s ** 0.5), ncross=4)
    return pool


def accuracy_check(srv, reqs, count=6, max_n=20000):
    """The largest |dS| between served results and FP64 solves of the same (board, frequency), over up to `count`
    requests on boards of at most max_n unknowns (a fresh double-precision solver on the default stream)."""
    from .operator import DirectSolver
    picks = [r for r in reqs if r.error is None and srv.size(r.board) <= max_n][:count]
    worst, solvers = 0.0, {}
    for r in picks:
        geo = srv._geometry(r.board)
        ds = solvers.setdefault(r.board, DirectSolver(geo))
        S = geo.sparams_from_currents(ds.solve_direct(r.f, geo.excitation(), precision='double').cpu().numpy(), r.f)
        ds.release()
        worst = max(worst, float(np.abs(S - r.S).max()))
    return worst, len(picks)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--rate', type=float, nargs='+', default=[20.0], help='arrival rates (req/s); several: a sweep')
    ap.add_argument('--requests', type=int, default=40)
    ap.add_argument('--slots', type=int, default=4)
    ap.add_argument('--seed', type=int, default=0)
    ap.add_argument('--targets', type=int, nargs='+', default=[2000, 5000, 10000, 20000, 40000])
    ap.add_argument('--weights', type=float, nargs='+', default=None)
    ap.add_argument('--check', type=int, default=6, help='served results checked against FP64 solves, per rate')
    a = ap.parse_args()
    import torch
    torch.cuda.set_device(0)
    pool = board_pool(a.seed, tuple(a.targets))
    keys = list(pool)
    weights = a.weights or [0.3, 0.3, 0.2, 0.15, 0.05][:len(keys)]
    srv = Server(pool, slots=a.slots)
    for k in keys:                                        # resident boards: geometry built before serving
        srv.size(k)
    srv.run([Request(-1 - j, k, 3e9, 0.0) for j, k in enumerate(keys)])       # first use of each board (untimed)
    for rate in a.rate:
        reqs = poisson_requests(keys, weights, rate, a.requests, seed=a.seed)
        srv.peak_bytes = 0.0
        t = time.perf_counter()
        srv.run(reqs)
        wall = time.perf_counter() - t
        out = dict(rate=rate, slots=a.slots, sizes={k: srv.size(k) for k in keys}, weights=weights, wall_s=round(wall, 3),
                   budget_gb=round(srv.budget / GB, 1), peak_held_gb=round(srv.peak_bytes / GB, 1))
        out.update(Server.report(reqs, wall))
        if a.check:
            dS, n = accuracy_check(srv, reqs, a.check)
            out.update(max_dS_vs_fp64=dS, checked=n)
        print(json.dumps(out), flush=True)


if __name__ == '__main__':
    main()
