"""
mom25d_b200.batch - one board's whole frequency sweep at once: every frequency an independent mixed-precision
solve, several in flight on one GPU, against the same frequencies solved one after another in FP64.

    python -m mom25d_b200.batch [--freqs 64] [--fmin 1e9] [--fmax 6e9] [--slots 6] [--fp64 64]

The workload is the stub filter board (board.stub_filter_board: three layers 0.2 / 1.0 / 0.2 mm, a 50 ohm line
40 mm long with an open quarter-wave stub at 2.4 GHz, dmax 0.2 mm, a via port at each line end) at
linspace(fmin, fmax, freqs).

  - batched: the Green tables of every frequency are built and kept on the device, and the far part of every
    frequency's double Z is filled by one launch (m25_fill_far_multi, grid z = frequency; in chunks where the
    matrices of all frequencies would not fit); then all frequencies are present at the start and go through the
    serving loop (serve.Server), each with its prefilled Z: each slot has its own CUDA stream, host thread and
    solver, which adds the near field and via border, factors and refines, so one frequency's panel
    factorisation, triangular solves and host synchronisations overlap the others' tensor-core updates. Kept-LU
    reuse is off (each frequency's result does not depend on the others');
  - sequential mixed: the reference's sweep (fast.py:996-1118) on one stream, kept complex64 LUs reused within the
    learnt reach;
  - FP64: the drop-in path, one frequency after another (each its own complex128 fill and LU).

Reported (one JSON line): solves/s of each (wall clock around the sweep, after a warm-up; the batched one the median
of three sweeps), the batched-over-FP64
ratio, and the largest |dS| of both mixed sweeps against FP64 over the frequencies FP64 solved.
"""
import argparse
import json
import time

import numpy as np

from .serve import Request, Server


def sweep_requests(key, freqs):
    """A sweep as requests that have all arrived at the start, in frequency order."""
    return [Request(i, key, f, 0.0) for i, f in enumerate(freqs)]


def fill_far_sweep(geo, dg, freqs, stream=None):
    """The far part of the double Z at every frequency in one launch (m25_fill_far_multi): each frequency's Green
    tables (device.DeviceTables) built and kept, one N x N complex128 Z a frequency. Returns (Zs, tables)."""
    import ctypes
    import torch
    from ._lib import P, check, lib, stream_ptr
    from .device import DeviceTables
    N = geo.N
    tabs = [DeviceTables(dg, f, stream=stream) for f in freqs]
    Zs = [torch.empty((N, N), dtype=torch.complex128, device='cuda') for _ in freqs]
    ptrs = torch.tensor([Z.data_ptr() for Z in Zs], dtype=torch.int64, device='cuda')
    raw = b''.join(ctypes.string_at(ctypes.addressof(t.tables), ctypes.sizeof(t.tables)) for t in tabs)
    d_tb = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to('cuda')
    d_w = torch.tensor([2 * np.pi * f for f in freqs], dtype=torch.float64, device='cuda')
    check(lib().m25_fill_far_multi(P(ptrs), ctypes.c_long(N), ctypes.c_int(0), ctypes.byref(dg.mesh), P(d_tb), P(d_w),
                                   ctypes.c_int(len(freqs)), stream_ptr(stream)), 'm25_fill_far_multi')
    (stream or torch.cuda.current_stream()).synchronize()
    return Zs, tabs


class _ChunkFill:
    """The far part of a sweep's Z filled chunk by chunk on a stream and host thread of its own, one launch a chunk
    (fill_far_sweep), while the serving loop solves the chunks already filled: request i's far() waits for its
    chunk, then hands over its Z (and lets go of it)."""

    def __init__(self, geo, dg, freqs, chunk):
        import threading
        import torch
        self.freqs, self.chunk = [float(f) for f in freqs], chunk
        self.ready = [threading.Event() for _ in range(0, len(freqs), chunk)]
        self.Z, self.error = {}, None
        self.stream = torch.cuda.Stream()
        self.thread = threading.Thread(target=self._run, args=(geo, dg), daemon=True)
        self.thread.start()

    def _run(self, geo, dg):
        import torch
        try:
            with torch.cuda.stream(self.stream):
                for c, c0 in enumerate(range(0, len(self.freqs), self.chunk)):
                    part = self.freqs[c0:c0 + self.chunk]
                    Zs, tabs = fill_far_sweep(geo, dg, part, stream=self.stream)
                    for i, Z in enumerate(Zs):
                        self.Z[c0 + i] = Z
                    del Zs, tabs
                    self.ready[c].set()
        except Exception as e:                     # the requests of the chunks not filled report it
            self.error = e
            for ev in self.ready:
                ev.set()

    def far(self, i):
        def get():
            self.ready[i // self.chunk].wait()
            if self.error is not None:
                raise RuntimeError(f"batched sweep: the far fill failed: {self.error}")
            return self.Z.pop(i)
        return get


def batched_sweep(server, key, freqs, multi=True, chunk=None):
    """All frequencies through the server at once: (S list in frequency order, wall seconds, requests). multi: the
    far part of every frequency's Z filled by one launch a chunk (default: a quarter of the sweep, as memory
    allows) on a stream of its own, overlapping the solves of the chunks before it, the requests carrying their Z;
    else each request fills its own."""
    t = time.perf_counter()
    if not multi:
        reqs = sweep_requests(key, freqs)
        server.run(reqs)
    else:
        import torch
        from .device import DeviceGeometry
        geo = server._geometry(key)
        dg = getattr(server, '_fill_dg', {}).get(key)
        if dg is None:
            dg = DeviceGeometry(geo)
            server._fill_dg = {key: dg}
        free, _ = torch.cuda.mem_get_info()
        per = 16.0 * geo.N * geo.N
        room = 0.8 * free - server.slots * (server.footprint(key) + 2e9)
        fits = max(1, int(room // per) // 2)                 # (two chunks in memory at once)
        chunk = max(1, min(chunk or -(-len(freqs) // 4), fits))
        filler = _ChunkFill(geo, dg, freqs, chunk)
        reqs = [Request(i, key, f, 0.0, far=filler.far(i)) for i, f in enumerate(freqs)]
        server.run(reqs)
        filler.thread.join()
    wall = time.perf_counter() - t
    bad = [r for r in reqs if r.error is not None]
    if bad:
        raise RuntimeError(f"batched sweep: {len(bad)} frequencies failed, the first: {bad[0].error}")
    return [r.S for r in reqs], wall, reqs


def sequential_sweep(sim, freqs):
    """One frequency after another through Simulation.sparams: (S list, wall seconds)."""
    import torch
    out = []
    torch.cuda.synchronize()
    t = time.perf_counter()
    for f in freqs:
        out.append(sim.sparams(f))
    torch.cuda.synchronize()
    return out, time.perf_counter() - t


def max_dS(A, B):
    return float(max(np.abs(np.asarray(a) - np.asarray(b)).max() for a, b in zip(A, B)))


def run(board, freqs, slots=6, fp64_count=None, sequential_mixed=True, reps=3):
    import torch
    from .sim import Simulation
    freqs = [float(f) for f in freqs]
    fp64_count = len(freqs) if fp64_count is None else min(int(fp64_count), len(freqs))
    key = getattr(board, 'name', 'board')
    srv = Server({key: board}, slots=slots)
    N = srv.size(key)
    # warm-up: a solve on every slot (kernels loaded, solvers, streams and buffers built)
    batched_sweep(srv, key, [freqs[len(freqs) // 2]] * slots)
    walls = []
    for _ in range(max(1, reps)):                         # the median of reps sweeps (one is about a second)
        S_b, wall_b, reqs = batched_sweep(srv, key, freqs)
        walls.append(wall_b)
    wall_b = float(np.median(walls))
    del srv._fill_dg
    out = dict(workload=f"{key}: N={N} unknowns, {len(freqs)} frequencies linspace({freqs[0] / 1e9:.4g}, "
                        f"{freqs[-1] / 1e9:.4g} GHz)", unknowns=N, frequencies=len(freqs), slots=slots,
               batched=dict(solves_per_s=round(len(freqs) / wall_b, 3), wall_s=round(wall_b, 3),
                            walls_s=[round(w, 3) for w in walls],
                            paths={p: sum(r.path == p for r in reqs) for p in sorted({r.path for r in reqs})}))
    del srv
    torch.cuda.empty_cache()
    fsel = freqs[:fp64_count] if fp64_count == len(freqs) else \
        [freqs[i] for i in np.linspace(0, len(freqs) - 1, fp64_count).round().astype(int)]
    isel = [freqs.index(f) for f in fsel]
    sim64 = Simulation.from_board(board, precision='double')
    sim64.sparams(fsel[0])                                # warm-up
    S_d, wall_d = sequential_sweep(sim64, fsel)
    out['fp64'] = dict(solves_per_s=round(len(fsel) / wall_d, 3), wall_s=round(wall_d, 3), frequencies=len(fsel))
    out['batched_over_fp64'] = round(out['batched']['solves_per_s'] / out['fp64']['solves_per_s'], 3)
    out['max_dS_batched_vs_fp64'] = max_dS([S_b[i] for i in isel], S_d)
    del sim64
    torch.cuda.empty_cache()
    if sequential_mixed:
        simm = Simulation.from_board(board, precision='mixed')
        simm.sparams(freqs[len(freqs) // 2])              # warm-up, then a cold sweep
        ds = simm.fast
        ds.forget()
        S_m, wall_m = sequential_sweep(simm, freqs)
        out['sequential_mixed'] = dict(solves_per_s=round(len(freqs) / wall_m, 3), wall_s=round(wall_m, 3))
        out['max_dS_sequential_mixed_vs_fp64'] = max_dS([S_m[i] for i in isel], S_d)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--freqs', type=int, default=64)
    ap.add_argument('--fmin', type=float, default=1e9)
    ap.add_argument('--fmax', type=float, default=6e9)
    ap.add_argument('--slots', type=int, default=6)
    ap.add_argument('--fp64', type=int, default=None, help='FP64 solves to time and compare (default: all)')
    ap.add_argument('--dmax', type=float, default=0.2e-3)
    ap.add_argument('--no-sequential-mixed', action='store_true')
    a = ap.parse_args()
    import torch
    from .board import stub_filter_board
    torch.cuda.set_device(0)
    bd = stub_filter_board(dmax=a.dmax)
    out = run(bd, np.linspace(a.fmin, a.fmax, a.freqs), slots=a.slots, fp64_count=a.fp64,
              sequential_mixed=not a.no_sequential_mixed)
    print(json.dumps(out))


if __name__ == '__main__':
    main()
