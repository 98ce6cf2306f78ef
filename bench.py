"""
bench.py - frequency solves per second on the ~20k-unknown seeded synthetic routed board (24 Manhattan traces,
16 vias, 8 via ports, 3-layer stack 0.2 / 1.0 / 0.2 mm), one step = one frequency: Green tables, fill, near
field, via border, LU, solve / refinement, S. Headline: the mixed-precision path (complex64 fill and LU refined to
the double-precision operator); beside it the FP64 drop-in path, |dS| between them, per-step p50 / p99 latency.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--fp64-steps K2] [--no-cpu-baseline]

Multi-GPU: replicas only (frequencies are independent; no collective on the data path): every rank solves its
own frequencies, the time is the max over ranks. --impl reference times the reference's CPU implementation of
the path (its compiled core built from source, oracle/_ref, and LAPACK through SciPy) on the host cores.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solved freqs/sec, 20k-unknown board: mixed-prec vs FP64 (|ΔS|≤1e-4); p50/p99 ms"
SEED, NCROSS = 1, 4
FREQS = np.geomspace(0.5e9, 10e9, 21)


def board():
    from mom25d_b200.board import routed_board
    return routed_board(seed=SEED, ncross=NCROSS)


def workload(geo):
    return {"workload": f"routed_board(seed={SEED}): 24 traces, 16 vias, 8 via ports, 3-layer stack, dmax 0.25 mm, "
                        f"N={geo.N} unknowns, {geo.Nt} triangles, f = geomspace(0.5, 10 GHz, 21)",
            "unknowns": int(geo.N), "ports": len(geo.ports), "l2": "inputs larger than L2 (Z is N^2 complex)"}


# ---- clocks during the timed region --------------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index, self.rows, self.proc = index, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.Q,
                                          '--format=csv,noheader,nounits', '-lms', '200'], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(',')])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(2)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace('.', '').isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9 for i in range(4) if r[5 + i] == 'Active'})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---- the reference's CPU path on a bounded sample -------------------------------------------------------------------
def cpu_reference(geo, n_lu=6000):
    """The reference's FP64 direct solve timed on this host's cores: its compiled core (oracle/_ref, built from its
    sources) for the far fill and near correction of the full board, LAPACK zgetrf / zgetrs through SciPy on a
    leading n_lu x n_lu block of Z (scaled by (N / n_lu)^3 to the full LU), the Green tables from the oracle's
    NumPy restatement of the reference's. Returns (freq solves / s, cores, sample description)."""
    import scipy.linalg as sla
    sys.path.insert(0, os.path.join(ROOT, 'oracle', '_ref'))
    import oracle
    from oracle import green, solve as osolve
    cores = len(os.sched_getaffinity(0))
    os.environ.setdefault('OMP_NUM_THREADS', str(cores))
    try:
        import _core as core
        kind = 'reference'
    except ImportError:
        core, kind = oracle, 'port'
    try:
        from threadpoolctl import threadpool_limits
        threadpool_limits(cores)
    except Exception:
        pass
    f = float(FREQS[10])
    P, Q = core.near_pairs(geo.g['cent'], geo.tri_size, geo.tri_z, geo.near_fac)
    P32, Q32 = P.astype(np.int32), Q.astype(np.int32)
    t = {}
    t0 = time.perf_counter()
    tables = green.green_tables(geo, f)
    tb = green.core_tables(geo, tables)
    t['tables'] = time.perf_counter() - t0
    N, w = geo.N, 2 * np.pi * f
    Z = np.zeros((N, N), complex)
    t0 = time.perf_counter()
    core.fill_far(Z, geo.g, tb, w)
    t['fill_far'] = time.perf_counter() - t0
    q = dict(geo.q, stat=np.zeros((len(P), 12)), stat_ready=False)
    t0 = time.perf_counter()
    core.near_into_dense(Z, geo.g, tb, q, P32, Q32, w)
    t['near'] = time.perf_counter() - t0
    n = min(n_lu, N)
    A = Z[:n, :n].copy()
    A += np.eye(n) * np.abs(np.diagonal(A)).max()            # (a well-posed block of the same size)
    t0 = time.perf_counter()
    F = sla.lu_factor(A.T, overwrite_a=True, check_finite=False)
    t_lu = time.perf_counter() - t0
    B = np.ones((n, len(geo.ports)), complex)
    t0 = time.perf_counter()
    sla.lu_solve(F, B, trans=1, check_finite=False)
    t_solve = time.perf_counter() - t0
    t['lu'] = t_lu * (N / n) ** 3
    t['solve'] = t_solve * (N / n) ** 2
    total = sum(t.values())
    sample = (f"one frequency ({f / 1e9:.3g} GHz) of the FP64 path: tables + far fill + near correction at full size "
              f"(N={N}); LU and solve timed at n={n} and scaled by (N/n)^3, (N/n)^2; seconds: " +
              ", ".join(f"{k} {v:.2f}" for k, v in t.items()))
    return 1.0 / total, cores, sample, kind, t


# ---- replicas: the frequency split and the max over ranks -----------------------------------------------------------
def rank_frequencies(rank, world):
    """This rank's frequencies: the sweep in a strided order (step i: FREQS[8 i mod 21]), so that a run of fewer
    than 21 steps samples the whole band rather than its low end; rank r takes every world-th from position r."""
    order = [float(FREQS[(8 * i) % len(FREQS)]) for i in range(len(FREQS))]
    return [f for i, f in enumerate(order) if i % world == rank]


def max_over_ranks(values, world, device):
    """Element-wise max of a list of floats over the ranks (the timing rule); the list itself at world = 1."""
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


# ---- the GPU arm ----------------------------------------------------------------------------------------------------
def run_gpu(args, rank, world):
    import torch
    import torch.distributed as dist
    from mom25d_b200 import _lib
    from mom25d_b200.sim import Simulation
    dev = int(os.environ.get('LOCAL_RANK', 0))
    torch.cuda.set_device(dev)
    bd = board()
    sim = Simulation.from_board(bd, precision='mixed')
    geo = sim.geo
    ds = sim.fast
    mine = rank_frequencies(rank, world)
    E_host = torch.from_numpy(geo.excitation()).pin_memory()
    E_dev = E_host.to('cuda')
    stream = torch.cuda.current_stream()

    def step_device(f, precision):
        """One frequency through the kernels, inputs resident: (ms, getrf ms)."""
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        if precision == 'mixed':
            sim.precision = 'mixed'
            X = sim.currents(f, E_dev)          # mixed, redone in double where the refinement fails (fast.py:844)
        else:
            X = ds.solve_direct(f, E_dev, precision='double')
        b.record(stream)
        b.synchronize()
        step_device.X = X
        return a.elapsed_time(b), (ds.last_lu_c64_ms if precision == 'mixed' else ds.last_lu_ms)

    # warm-up (also the accuracy check: mixed vs double at one frequency)
    for i in range(args.warmup):
        step_device(mine[i % len(mine)], 'mixed')
    fchk = mine[len(mine) // 2]
    X_m = ds.solve_direct(fchk, E_dev, precision='mixed')
    res_m = float(np.max(ds.residual))
    S_m = geo.sparams_from_currents(X_m.cpu().numpy())
    X_d = ds.solve_direct(fchk, E_dev, precision='double')
    S_d = geo.sparams_from_currents(X_d.cpu().numpy())
    dS = float(np.abs(S_m - S_d).max())
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    lib = _lib.lib()
    lib.m25_launch_count.restype = ctypes.c_longlong
    n0 = lib.m25_launch_count()
    clk = Clocks(dev)
    clk.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    def cold():
        """A sweep starts with no kept LUs and nothing learnt (the warm-up and the accuracy check above left some)."""
        ds.kept, ds.reach, ds.t_iter, ds.mixed_failed = [], float(np.log(2.0)), None, 0.0

    cold()
    lat, lu_ms, iters, paths, kept_X = [], [], [], {}, []
    ds.timings, ds.attempts = {}, []
    for i in range(args.steps):
        ms, lms = step_device(mine[i % len(mine)], 'mixed')
        lat.append(ms); iters.append(max(ds.iters) if ds.iters else 0)
        if lms is not None:
            lu_ms.append(lms)
        paths[ds.last_path] = paths.get(ds.last_path, 0) + 1
        if args.verbose:
            print(f"step {i}: {mine[i % len(mine)] / 1e9:.4g} GHz {ds.last_path:22s} {iters[-1]:3d} iterations "
                  f"{ms:8.1f} ms", file=sys.stderr)
    attempts = list(ds.attempts)
    if args.verbose:
        for a in attempts:
            print(f"reuse {a['f'] / 1e9:.4g} GHz from {a['f0'] / 1e9:.4g}: cap {a['cap']}, {a['iters']} iterations, "
                  f"{'converged' if a['ok'] else 'not converged'} ({a['rel']:.1e})", file=sys.stderr)
        if i < args.fp64_steps:
            kept_X.append(step_device.X)        # compared with the FP64 solve of the same frequency below
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    launches = lib.m25_launch_count() - n0
    t_dev = ev0.elapsed_time(ev1) / 1000.0
    phases = {k: round(1000 * v / args.steps, 2) for k, v in ds.timings.items()}
    # FP64 drop-in path
    lat64, lu64 = [], []
    for i in range(args.fp64_steps):
        ms, lms = step_device(mine[i % len(mine)], 'double')
        lat64.append(ms); lu64.append(lms)
        if i < len(kept_X):
            S_m = geo.sparams_from_currents(kept_X[i].cpu().numpy())
            S_d = geo.sparams_from_currents(step_device.X.cpu().numpy())
            dS = max(dS, float(np.abs(S_m - S_d).max()))
    kept_X.clear()
    # end to end through the public API: E from pinned host memory, the port currents back, S on the host
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cold()
    e0.record(stream)
    for i in range(args.steps):
        sim.sparams(mine[i % len(mine)])
    e1.record(stream)
    torch.cuda.synchronize()
    t_e2e = e0.elapsed_time(e1) / 1000.0
    t_dev, t_e2e, t64 = max_over_ranks([t_dev, t_e2e, sum(lat64) / 1000.0], world, 'cuda')
    if rank != 0:
        return None
    N = geo.N
    flops_lu = 8.0 / 3.0 * N ** 3
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, 'MEASURED_PEAKS.json')))
    except Exception:
        pass
    tensor_peak = peaks.get('bf16_tflops_sustained', 1400.0)
    lu_avg = statistics.mean(lu_ms) / 1000.0 if lu_ms else float('nan')
    achieved = flops_lu / lu_avg / 1e12 if lu_ms else 0.0
    value = world * args.steps / t_dev
    e2e = world * args.steps / t_e2e
    fp64 = (world * args.fp64_steps / t64) if args.fp64_steps else None
    bytes_h2d = int(E_host.numel() * 16)
    bytes_d2h = int(len(sim.port_rows()[0]) * E_host.shape[1] * 16)
    traffic = None                           # DRAM bytes of one complex64 factorisation, from an ncu capture
    try:
        cap = json.load(open(os.path.join(ROOT, 'profiles', 'traffic.json')))['complex64_lu']
        if int(cap['n']) == N:
            traffic = cap['bytes_per_factorisation']
    except Exception:
        pass
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "freq-solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1000 * t_dev / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64+tf32x3/f64" if ds.tf32 else "c64/f64",
        "data": "synthetic (seeded routed board)", "config": workload(geo),
        "p50_ms": round(float(np.percentile(lat, 50)), 3), "p99_ms": round(float(np.percentile(lat, 99)), 3),
        "fp64": {"value": round(fp64, 4) if fp64 else None, "steps": args.fp64_steps,
                 "p50_ms": round(float(np.percentile(lat64, 50)), 3) if lat64 else None,
                 "lu_ms": round(statistics.mean(lu64), 3) if lu64 else None},
        "mixed_over_fp64": round(value / fp64, 3) if fp64 else None,
        "max_dS_mixed_vs_fp64": dS, "mixed_rel_residual": res_m, "gmres_iters_max": int(max(iters)),
        "lu_ms": round(1000 * lu_avg, 3) if lu_ms else None, "factorisations": len(lu_ms), "paths": paths,
        "reuse_attempts": {"tried": len(attempts), "converged": sum(1 for a in attempts if a['ok'])},
        "phases_ms_per_step": phases,
        "e2e": {"value": round(e2e, 4), "unit": "freq-solves/s", "h2d_bytes_per_step": bytes_h2d,
                "d2h_bytes_per_step": bytes_d2h},
        "gpu_launches": int(launches),
        "roofline": {"kernel": "complex64 LU with 3xTF32 tcgen05 updates (m25_getrf), 8/3 N^3 flops a factorisation",
                     "bound": "tensor", "achieved": round(achieved, 2), "peak": tensor_peak, "unit": "TFLOP/s",
                     "frac": round(achieved / tensor_peak, 4), "traffic": traffic,
                     "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained" if peaks else "fallback"},
        "clocks": clocks,
    }
    if not args.no_cpu_baseline and world == 1:
        v, cores, sample, kind, _ = cpu_reference(geo)
        line["cpu_baseline"] = {"value": round(v, 5), "unit": "freq-solves/s", "cores": cores, "kind": kind,
                                "sample": sample}
    return line


def run_reference(args, rank, world):
    """The reference arm: its CPU implementation of the path on this host (rank 0 only)."""
    if rank != 0:
        return None
    from mom25d_b200.geometry import Geometry
    geo = Geometry(board())
    vals = []
    for i in range(args.warmup + args.steps):
        v, cores, sample, kind, _ = cpu_reference(geo, n_lu=args.ref_lu)
        if i >= args.warmup:
            vals.append(v)
    v = statistics.median(vals)
    return {"impl": "reference", "metric": METRIC, "value": round(v, 5), "unit": "freq-solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 / v, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded routed board)",
            "config": workload(geo),
            "cpu_baseline": {"value": round(v, 5), "unit": "freq-solves/s", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(v, 5), "unit": "freq-solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=21)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--fp64-steps', type=int, default=3)
    ap.add_argument('--impl', default='b200')
    ap.add_argument('--ref-lu', type=int, default=6000)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--verbose', action='store_true', help='each timed step and reuse attempt on stderr')
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank, world = int(os.environ.get('RANK', 0)), int(os.environ.get('WORLD_SIZE', 1))
    if args.impl == 'reference':
        line = run_reference(args, rank, world)
    else:
        import torch.distributed as dist
        if world > 1:
            import datetime
            import torch
            torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', 0)))
            dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600))
        try:
            line = run_gpu(args, rank, world)
        finally:
            if world > 1:
                dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == '__main__':
    main()
