"""
bench.py - frequency solves per second on the ~20k-unknown seeded synthetic routed board (24 Manhattan traces,
16 vias, 8 via ports, 3-layer stack 0.2 / 1.0 / 0.2 mm), one step = one frequency: Green tables, fill, near
field, via border, LU, solve / refinement, S. Headline: the mixed-precision path (complex64 fill and LU refined to
the double-precision operator); beside it the FP64 drop-in path, |dS| between them, per-step p50 / p99 latency.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--fp64-steps K2] [--no-cpu-baseline]

Every timed step is checked after the timed region against the FP64 drop-in at its frequency (|dS|, and the
normwise backward error of the mixed currents in the double-precision Z); the FP64 solves are timed over the same
frequencies. The FP64 path is also checked against the reference's CPU path at one frequency (Z and S).

Multi-GPU: replicas only (frequencies are independent; no collective on the data path): every rank solves its
own frequencies, the time is the max over ranks. --impl reference times the reference's CPU implementation of
the path (its compiled core built from source, oracle/_ref, and LAPACK through SciPy) on the host cores, on its
default path at this size (mixed precision, kept complex64 LUs), at full size.
"""
import argparse
import ctypes
import gc
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


# ---- the reference's CPU path ----------------------------------------------------------------------------------------
def _ref_core():
    """The reference's compiled core (oracle/_ref, built from its sources) and its kind; the oracle's C restatement
    of it where that was not built."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle', '_ref'))
    try:
        import _core
        return _core, 'reference'
    except ImportError:
        import oracle
        return oracle, 'port'


def _cpu_threads():
    cores = len(os.sched_getaffinity(0))
    os.environ.setdefault('OMP_NUM_THREADS', str(cores))
    try:
        from threadpoolctl import threadpool_limits
        threadpool_limits(cores)
    except Exception:
        pass
    return cores


def cpu_sweep(geo, freqs, precision='mixed', sweep=None):
    """The reference's CPU path over `freqs`, one frequency after another at full size (no extrapolation): its
    compiled core for the far fill and near correction, the Green tables and via blocks of the oracle's NumPy
    restatement, LAPACK through SciPy; precision 'mixed' is the reference's default above 3,500 unknowns
    (sim.py:61): double Z, complex64 LUs kept and reused across frequencies, GMRES with dense double products
    (fast.py:704-850, 996-1084). Returns (seconds per frequency, paths, the sweep object)."""
    from oracle import solve as osolve
    core, _ = _ref_core()
    ks = sweep or osolve.KeptSweep(geo, core=core)
    secs, paths = [], []
    for f in freqs:
        t = time.perf_counter()
        ks.solve(float(f), precision=precision)
        secs.append(time.perf_counter() - t)
        paths.append(ks.last_path)
    return secs, paths, ks


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
def backward_errors(ds, Z, X, E):
    """Normwise backward error of each column of X for Z X = E (Rigal and Gaches): |E - Z X|_inf / (|Z|_inf
    |X|_inf + |E|_inf); Z the unequilibrated double-precision matrix on the device (row-major N x N)."""
    import torch
    R = E - ds._dense(Z, X)
    zn = float(Z.abs().sum(dim=1).max())
    rn = R.abs().amax(dim=0)
    xn = X.abs().amax(dim=0)
    en = E.abs().amax(dim=0)
    return (rn / (zn * xn + en)).cpu().numpy()


def fp64_vs_reference(ds, geo, f, E_dev, sweep):
    """The FP64 drop-in against the reference's CPU path at one frequency: Z relative Frobenius difference (the
    reference's Z uploaded and compared on the device), and S from the reference's double LU (LAPACK zgetrf) vs
    S of the FP64 GPU solve; plus the reference's mixed solve, whose time is the CPU baseline. Returns (parity
    dict, the CPU mixed solve's seconds, its phase seconds)."""
    import torch
    Zg = ds.impedance(f, 'double')
    sweep.timings = {}
    t = time.perf_counter()
    Zc = sweep.impedance(f)
    t_fill = time.perf_counter() - t
    Zc_dev = torch.from_numpy(Zc).to('cuda')
    z_rel = float(torch.linalg.norm(Zg - Zc_dev) / torch.linalg.norm(Zc_dev))
    del Zc_dev
    E = geo.excitation()
    t = time.perf_counter()
    Xm_cpu = sweep.solve_z(f, Zc, E, precision='mixed')
    t_mixed = t_fill + time.perf_counter() - t
    phases = dict(sweep.timings)
    del Zc
    Zc = sweep.impedance(f)
    Xd_cpu = sweep.solve_z(f, Zc, E, precision='double')
    del Zc
    Xd_gpu = ds.solve_direct(f, E_dev, precision='double').cpu().numpy()
    S_ref, S_gpu = geo.sparams_from_currents(Xd_cpu), geo.sparams_from_currents(Xd_gpu)
    S_refm = geo.sparams_from_currents(Xm_cpu)
    out = {"f_ghz": round(f / 1e9, 4), "z_rel_fro": z_rel, "max_dS_fp64_gpu_vs_reference": float(np.abs(S_gpu - S_ref).max()),
           "max_dS_reference_mixed_vs_its_fp64": float(np.abs(S_refm - S_ref).max()),
           "bar": "Z rel-Frobenius <= 1e-10, max |dS| <= 1e-8"}
    return out, t_mixed, phases


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
        """One frequency through the kernels, inputs resident: (ms, getrf ms, currents)."""
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        if precision == 'mixed':
            sim.precision = 'mixed'
            X = sim.currents(f, E_dev)          # mixed, redone in double where the refinement fails (fast.py:844)
        else:
            X = ds.solve_direct(f, E_dev, precision='double')
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b), (ds.last_lu_c64_ms if precision == 'mixed' else ds.last_lu_ms), X

    def cold():
        """A sweep starts with no kept LUs and nothing learnt (the warm-up leaves some)."""
        ds.forget()

    for i in range(args.warmup):
        step_device(mine[i % len(mine)], 'mixed')
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    lib = _lib.lib()
    n0 = lib.m25_launch_count()
    clk = Clocks(dev)
    clk.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cold()
    lat, lu_ms, iters, paths, kept_X, step_path = [], [], [], {}, [], []
    ds.timings, ds.attempts = {}, []
    gc.collect()
    gc.disable()                            # no collector pause inside a timed region (as timeit does)
    ev0.record(stream)
    for i in range(args.steps):
        ph0 = dict(ds.timings) if args.verbose else None
        ms, lms, X = step_device(mine[i % len(mine)], 'mixed')
        lat.append(ms); iters.append(max(ds.iters) if ds.iters else 0)
        if lms is not None:
            lu_ms.append(lms)
        paths[ds.last_path] = paths.get(ds.last_path, 0) + 1
        step_path.append(ds.last_path)
        kept_X.append(X)                    # compared with the FP64 solve of the same frequency below
        if args.verbose:
            rh = getattr(ds, 'res_hist', [])
            ph = {k: 1000 * (v - ph0.get(k, 0.0)) for k, v in ds.timings.items() if v - ph0.get(k, 0.0) > 5e-4}
            print(f"step {i}: {mine[i % len(mine)] / 1e9:.4g} GHz {ds.last_path:22s} {iters[-1]:3d} iterations "
                  f"{ms:8.1f} ms  phases " + ' '.join(f"{k} {v:.0f}" for k, v in ph.items()) +
                  "  residual by step: " + ' '.join(f"{x:.0e}" for x in rh[1::3]), file=sys.stderr)
    ev1.record(stream)
    torch.cuda.synchronize()
    gc.enable()
    clocks = clk.stop()
    launches = lib.m25_launch_count() - n0
    t_dev = ev0.elapsed_time(ev1) / 1000.0
    phases = {k: round(1000 * v / args.steps, 2) for k, v in ds.timings.items()}
    attempts = list(ds.attempts)
    if args.verbose:
        for a in attempts:
            print(f"reuse {a['f'] / 1e9:.4g} GHz from {a['f0'] / 1e9:.4g}: cap {a['cap']}, {a['iters']} iterations, "
                  f"{'converged' if a['ok'] else 'not converged'} ({a['rel']:.1e})", file=sys.stderr)
    # every timed step against the FP64 drop-in at its frequency: |dS| and the mixed solution's backward error in
    # the double-precision Z; the FP64 solves themselves are the FP64 timing (over the same frequencies)
    dS, berr, lat64, lu64 = [], [], [], []
    n64 = args.steps if args.fp64_steps is None else min(args.fp64_steps, args.steps)
    for i in range(args.steps):
        f = mine[i % len(mine)]
        Z = ds.impedance(f, 'double')
        berr.append(float(backward_errors(ds, Z, kept_X[i], E_dev).max()))
        if i < n64:
            ms, lms, Xd = step_device(f, 'double')
            lat64.append(ms); lu64.append(lms)
        else:
            Xd = ds.solve_direct(f, E_dev, precision='double')
        S_m = geo.sparams_from_currents(kept_X[i].cpu().numpy())
        S_d = geo.sparams_from_currents(Xd.cpu().numpy())
        dS.append(float(np.abs(S_m - S_d).max()))
    kept_X.clear()
    # end to end through the public API: E from pinned host memory, the port currents back, S on the host
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cold()
    gc.collect()
    gc.disable()
    e0.record(stream)
    for i in range(args.steps):
        sim.sparams(mine[i % len(mine)])
    e1.record(stream)
    torch.cuda.synchronize()
    gc.enable()
    t_e2e = e0.elapsed_time(e1) / 1000.0
    solve_ms = time_solve_pair(ds, E_dev.shape[1])
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
    fp64 = (world * len(lat64) / t64) if lat64 else None
    bytes_h2d = int(E_host.numel() * 16)
    bytes_d2h = int(len(geo.port_rows()) * E_host.shape[1] * 16)
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
        "fp64": {"value": round(fp64, 4) if fp64 else None, "steps": len(lat64),
                 "p50_ms": round(float(np.percentile(lat64, 50)), 3) if lat64 else None,
                 "lu_ms": round(statistics.mean(lu64), 3) if lu64 else None,
                 "frequencies": "the timed mixed steps' own"},
        "mixed_over_fp64": round(value / fp64, 3) if fp64 else None,
        "max_dS_mixed_vs_fp64": max(dS), "max_backward_error_mixed": max(berr),
        "per_step": {"f_ghz": [round(mine[i % len(mine)] / 1e9, 4) for i in range(args.steps)], "path": step_path,
                     "ms": [round(x, 2) for x in lat], "gmres_iters": iters, "dS_vs_fp64": [float('%.3g' % x) for x in dS],
                     "backward_error": [float('%.3g' % x) for x in berr]},
        "lu_ms": round(1000 * lu_avg, 3) if lu_ms else None, "factorisations": len(lu_ms), "paths": paths,
        "reuse_attempts": {"tried": len(attempts), "converged": sum(1 for a in attempts if a['ok'])},
        "kept_lus_max": int(ds._keep_max()),
        "phases_ms_per_step": phases,
        "e2e": {"value": round(e2e, 4), "unit": "freq-solves/s", "h2d_bytes_per_step": bytes_h2d,
                "d2h_bytes_per_step": bytes_d2h},
        "gpu_launches": int(launches),
        "roofline": {"kernel": "complex64 LU with 3xTF32 tcgen05 updates (m25_getrf), 8/3 N^3 flops a factorisation",
                     "bound": "tensor", "achieved": round(achieved, 2), "peak": tensor_peak, "unit": "TFLOP/s",
                     "frac": round(achieved / tensor_peak, 4), "traffic": traffic,
                     "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained" if peaks else "fallback"},
        "roofline_fill": fill_roofline(geo, phases.get('fill')),
        "roofline_solve": solve_roofline(N, solve_ms, E_dev.shape[1], peaks.get('hbm_gbs')),
        "clocks": clocks,
        "host": "Python's garbage collector off inside the timed regions (collected before each)",
    }
    if not args.no_cpu_baseline and world == 1:
        from oracle import solve as osolve
        core, kind = _ref_core()
        cores = _cpu_threads()
        f_ref = float(FREQS[10])
        parity, t_cpu, cph = fp64_vs_reference(ds, geo, f_ref, E_dev, osolve.KeptSweep(geo, core=core))
        line["fp64_vs_reference"] = parity
        line["cpu_baseline"] = {"value": round(1.0 / t_cpu, 5), "unit": "freq-solves/s", "cores": cores, "kind": kind,
                                "sample": f"one frequency ({f_ref / 1e9:.3g} GHz) of the reference's default path "
                                          f"at this size (double Z, fresh complex64 LU, GMRES on the dense double Z; "
                                          f"fast.py:704-850, 996-1084) at full size, N={N}; seconds: " +
                                          ", ".join(f"{k} {v:.2f}" for k, v in cph.items())}
    return line


def time_solve_pair(ds, k, reps=10):
    """Device time (ms) of one complex64 solve pair (m25_getrs_aux: U^T then L^T, k right-hand sides) with the most
    recently kept complex64 factor: the median of `reps` after 3 untimed, CUDA events on the solver's stream."""
    import torch
    from mom25d_b200 import _lib
    if not ds.kept:
        return None
    rec = ds.kept[-1][1]
    N = rec['Z'].shape[0]
    L, st = _lib.lib(), ds.s
    g = torch.Generator(device='cuda').manual_seed(3)
    R = torch.complex(torch.randn(N, k, generator=g, device='cuda'), torch.randn(N, k, generator=g, device='cuda'))
    X = R.clone()
    stream = ds.stream if ds.stream is not None else torch.cuda.current_stream()
    times = []
    for i in range(3 + reps):
        X.copy_(R)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        _lib.check(L.m25_getrs_aux(_lib.P(rec['Z']), ctypes.c_long(N), ctypes.c_int(N), ctypes.c_int(1),
                                   _lib.P(rec['aux']), _lib.P(X), ctypes.c_int(k), st), 'm25_getrs_aux')
        b.record(stream)
        b.synchronize()
        if i >= 3:
            times.append(a.elapsed_time(b))
    _lib.sync_check(ds.stream)
    return statistics.median(times)


# FP64 flops of the fill per Z entry (edge tiles: 56 an entry + 30 a kernel evaluation, 0.95 evaluations an entry)
FILL_FLOPS_PER_ENTRY = 56 + 30 * 0.95
FP64_PEAK_TFLOPS = 36.6                  # a loop of independent FP64 FMAs over 148 x 8 CTAs of 256 threads, this B200


def fill_roofline(geo, fill_ms):
    """The fill's roofline (far fill + near correction, double precision, once a step): Ne^2 entries x 84.5 flops
    against the FP64 FMA rate measured on this pool's B200 (no FP64 figure in MEASURED_PEAKS.json)."""
    if not fill_ms:
        return None
    achieved = geo.Ne ** 2 * FILL_FLOPS_PER_ENTRY / (fill_ms / 1000.0) / 1e12
    return {"kernel": "far fill + near correction in FP64 (m25_fill_far, m25_near), Ne^2 x 84.5 flops a fill",
            "bound": "fp64", "achieved": round(achieved, 2), "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s",
            "frac": round(achieved / FP64_PEAK_TFLOPS, 4), "ms": fill_ms,
            "peak_source": "FP64 FMA loop measured on this pool's B200 (not in MEASURED_PEAKS.json)"}


def solve_roofline(N, ms, k, hbm):
    """The complex64 solve pair's roofline: the factor's two triangles (8 N^2 bytes) plus, at N >= 2,048, the 256-row
    blocks' inverses and couplings (2 x 3 x 256^2 complex64 entries a block), read once a pair, against HBM."""
    if not ms or not hbm:
        return None
    ns = -(-N // 256)
    nbytes = 8.0 * N * N + (6.0 * ns * 256 * 256 * 8 if N >= 2048 else 0.0)
    achieved = nbytes / (ms / 1000.0) / 1e9
    return {"kernel": f"complex64 solve pair with {k} right-hand sides (m25_getrs_aux)", "bound": "hbm",
            "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
            "ms_per_pair": round(ms, 3), "peak_source": "MEASURED_PEAKS.json hbm_gbs"}


def run_reference(args, rank, world):
    """The reference arm: the reference's CPU implementation of the path on this host (rank 0 only), on its
    default path at this size (mixed precision with kept complex64 LUs), the same strided frequency order and cold
    start as the GPU arm, every frequency at full size."""
    if rank != 0:
        return None
    from mom25d_b200.geometry import Geometry
    core, kind = _ref_core()
    cores = _cpu_threads()
    geo = Geometry(board())
    order = rank_frequencies(0, 1)
    freqs = [order[i % len(order)] for i in range(args.steps)]
    _, _, ks = cpu_sweep(geo, [order[i % len(order)] for i in range(args.warmup)])
    from oracle import solve as osolve
    ks = osolve.KeptSweep(geo, core=core)                 # cold, as the GPU arm's timed sweep
    secs, paths, ks = cpu_sweep(geo, freqs, sweep=ks)
    t_sum = sum(secs)
    v = args.steps / t_sum
    d_secs, _, _ = cpu_sweep(geo, freqs[:1], precision='double')
    phases = {k: round(1000 * x / args.steps, 1) for k, x in ks.timings.items()}
    sample = (f"the reference's default path at this size (mixed: double Z, complex64 LUs kept and reused, GMRES on "
              f"the dense double Z; fast.py:704-850, 996-1084) over {args.steps} frequencies of the sweep at full size "
              f"(N={geo.N}), no extrapolation; paths {dict((p, paths.count(p)) for p in set(paths))}; ms per step: "
              + ", ".join(f"{k} {x}" for k, x in phases.items()))
    return {"impl": "reference", "metric": METRIC, "value": round(v, 5), "unit": "freq-solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * t_sum / args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64 LU + c128 refinement",
            "data": "synthetic (seeded routed board)", "config": workload(geo),
            "p50_ms": round(1000 * float(np.percentile(secs, 50)), 1),
            "p99_ms": round(1000 * float(np.percentile(secs, 99)), 1),
            "fp64": {"value": round(1.0 / d_secs[0], 5), "steps": 1, "note": "the reference's double path (zgetrf)"},
            "cpu_baseline": {"value": round(v, 5), "unit": "freq-solves/s", "cores": cores, "kind": kind,
                             "sample": sample},
            "e2e": {"value": round(v, 5), "unit": "freq-solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=21)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--fp64-steps', type=int, default=None, help='FP64 solves timed (default: every timed step)')
    ap.add_argument('--impl', default='b200')
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
