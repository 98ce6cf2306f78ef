"""
mom25d_b200.tune - the autotuner of the LU's tile parameters, and timings of the hot path's kernels on this GPU.

    python -m mom25d_b200.tune --autotune [--sizes 2000 5000 10000 20000 40000] [--write]
    python -m mom25d_b200.tune --lu 8192 [--single] [--tf32] [--reps 3]     # the LU alone, CUDA events
    python -m mom25d_b200.tune --update 4096 4096 256                        # the tensor-core trailing update
    python -m mom25d_b200.tune --solve 18788 [--single]                      # the triangular solves, 8 columns
    python -m mom25d_b200.tune --dense 18788 8                               # the dense double product

Times are CUDA-event measurements on the launching stream after a warm-up, the matrix a random complex one with a
dominant diagonal (pivots away from it as well).

The autotuner times the LU at each size over its host-side parameters and keeps the fastest: for the complex64
LU with tensor-core updates (the mixed path's factorisation) the number of CTAs of the cooperative panel kernel
(16 to 64), its outer panel width kept at 256 columns - a narrower one leaves more of the factor's updates to
3xTF32 instead of FP32 and costs the factor its use as a preconditioner at the low-frequency end (measured on the
routed board: with 128, the fresh factor at 0.67 GHz no longer converged); for the complex128 LU (the drop-in)
both the outer panel width (128 / 192 / 256) and the panel CTAs. The winners per size go into TUNING_FILE
({"device", "sms", "complex64": [{"n", "nb2", "blocks", "ms"}], "complex128": [...]}), which the library reads at
load (_lib.apply_tuning -> m25_set_lu_tuning): a factorisation takes the entry nearest its size. The tensor-core
kernel's stage count is a compile-time choice (two stages, two CTAs an SM) and is not searched.
"""
import os
import argparse
import ctypes
import json
import time

import numpy as np
import torch

from . import _lib
from ._lib import P, check, lib


def random_matrix(n, dtype, seed=0):
    g = torch.Generator(device='cuda').manual_seed(seed)
    rdt = torch.float32 if dtype == torch.complex64 else torch.float64
    Z = torch.complex(torch.randn(n, n, generator=g, device='cuda', dtype=rdt),
                      torch.randn(n, n, generator=g, device='cuda', dtype=rdt))
    Z.diagonal().add_(4 * n ** 0.5)
    return Z


TUNING_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'tuning_b200.json')
GRIDS = {True: [(256, bl) for bl in (16, 24, 32, 48, 64)],
         False: [(b2, bl) for b2 in (128, 192, 256) for bl in (16, 32, 48)]}


def set_table(entries, single=True):
    """The LU's tuning table in the library: [(n, nb2, blocks)] for complex64 (single) or complex128."""
    arr = lambda i: (ctypes.c_int * max(1, len(entries)))(*[e[i] for e in entries])
    check(lib().m25_set_lu_tuning(int(single), arr(0), arr(1), arr(2), len(entries)), 'm25_set_lu_tuning')


def autotune(sizes, single=True, reps=2, log=print):
    """The fastest (nb2, blocks) per size for the complex64 (tensor-core) or complex128 LU:
    [{n, nb2, blocks, ms, grid: {"nb2/blocks": ms}}]."""
    out = []
    for n in sizes:
        grid = GRIDS[single]
        if n > 30000:                                     # (the largest size: a coarser grid, each LU is seconds)
            grid = [g for g in grid if g[1] in (32, 48)][:4]
        times = {}
        for b2, bl in grid:
            set_table([(1, b2, bl)], single)
            times[f"{b2}/{bl}"] = time_lu(n, single=single, tf32=single, reps=reps)['ms']
        best = min(times, key=times.get)
        b2, bl = map(int, best.split('/'))
        out.append(dict(n=int(n), nb2=b2, blocks=bl, ms=round(times[best], 2), grid={k: round(v, 2) for k, v in
                                                                                     times.items()}))
        if log:
            log(f"{'complex64' if single else 'complex128'} n={n}: nb2 {b2}, panel blocks {bl}: {times[best]:.1f} ms "
                f"(default 256/32: {times.get('256/32', float('nan')):.1f} ms)")
    set_table([(e['n'], e['nb2'], e['blocks']) for e in out], single)
    return out


def write_tuning(c64, c128, path=TUNING_FILE):
    import torch
    props = torch.cuda.get_device_properties(0)
    keep = lambda es: [{k: e[k] for k in ('n', 'nb2', 'blocks', 'ms')} for e in es]
    doc = dict(device=props.name, sms=props.multi_processor_count, complex64=keep(c64), complex128=keep(c128))
    with open(path, 'w') as fh:
        json.dump(doc, fh, indent=1)
    return path


def time_lu(n, single=False, tf32=False, reps=3):
    dtype = torch.complex64 if single else torch.complex128
    Z0 = random_matrix(n, dtype)
    Z = torch.empty_like(Z0)
    ipiv = torch.empty(n, dtype=torch.int32, device='cuda')
    nb = int(lib().m25_getrf_workspace(n, int(single)))
    work = torch.empty(nb, dtype=torch.uint8, device='cuda')
    out = []
    for r in range(reps + 1):
        Z.copy_(Z0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s = torch.cuda.current_stream()
        a.record(s)
        check(lib().m25_getrf(P(Z), ctypes.c_long(n), n, P(ipiv), int(single), int(tf32), P(work), ctypes.c_size_t(nb),
                              _lib.stream_ptr()), 'm25_getrf')
        b.record(s)
        _lib.sync_check()
        if r:
            out.append(a.elapsed_time(b))
    ms = float(np.median(out))
    flops = 8.0 / 3.0 * n ** 3
    return dict(n=n, single=single, tf32=tf32, ms=ms, tflops=flops / ms / 1e9)


def time_update(M, N, K, reps=5):
    """The complex64 trailing update C -= L U alone: tensor cores (3xTF32) and, for comparison, the LU's SIMT
    kernel through a factorisation-free call are both timed with CUDA events. 8 M N K flops."""
    ld = max(M, K)
    C = random_matrix(max(ld, N), torch.complex64)[:N, :].contiguous()          # N columns of ld
    L = random_matrix(max(ld, K), torch.complex64, seed=1)[:K, :].contiguous()
    U = random_matrix(max(ld, N), torch.complex64, seed=2)[:N, :].contiguous()
    nb = int((2 * 2 * M * 512 + 2 * N * 512) * 4 + 4096)
    work = torch.empty(nb, dtype=torch.uint8, device='cuda')
    s = torch.cuda.current_stream()
    out = []
    for r in range(reps + 1):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        check(lib().m25_cgemm_update_tf32(P(C), ctypes.c_long(C.shape[1]), M, N, K, P(L), P(U), P(work),
                                          ctypes.c_size_t(nb), _lib.stream_ptr()), 'm25_cgemm_update_tf32')
        b.record(s)
        _lib.sync_check()
        if r:
            out.append(a.elapsed_time(b))
    ms = float(np.median(out))
    return dict(M=M, N=N, K=K, ms=ms, tflops_complex=8.0 * M * N * K / ms / 1e9,
                tflops_tf32_issued=3 * 8.0 * M * N * K / ms / 1e9)


def time_solve(n, nrhs=8, single=True, reps=5):
    """The triangular solves with a factor (m25_getrs_aux, diagonal-block inverses prepared once)."""
    dtype = torch.complex64 if single else torch.complex128
    Z = random_matrix(n, dtype)
    ipiv = torch.empty(n, dtype=torch.int32, device='cuda')
    nb = int(lib().m25_getrf_workspace(n, int(single)))
    work = torch.empty(nb, dtype=torch.uint8, device='cuda')
    check(lib().m25_getrf(P(Z), ctypes.c_long(n), n, P(ipiv), int(single), int(single), P(work), ctypes.c_size_t(nb),
                          _lib.stream_ptr()), 'm25_getrf')
    na = int(lib().m25_getrs_aux_bytes(n, int(single)))
    aux = torch.empty(na, dtype=torch.uint8, device='cuda')
    check(lib().m25_getrs_prepare(P(Z), ctypes.c_long(n), n, P(ipiv), int(single), P(aux), ctypes.c_size_t(na),
                                  _lib.stream_ptr()), 'm25_getrs_prepare')
    B = random_matrix(max(n, nrhs), dtype, seed=3)[:n, :nrhs].contiguous()
    s = torch.cuda.current_stream()
    out = []
    for r in range(reps + 1):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        check(lib().m25_getrs_aux(P(Z), ctypes.c_long(n), n, int(single), P(aux), P(B), nrhs, _lib.stream_ptr()),
              'm25_getrs_aux')
        b.record(s)
        _lib.sync_check()
        if r:
            out.append(a.elapsed_time(b))
    ms = float(np.median(out))
    return dict(n=n, nrhs=nrhs, single=single, ms=ms, factor_GBps=n * n * (8 if single else 16) / ms / 1e6)


def time_dense(n, k=8, reps=5):
    """The refinement's dense double product Y = Z X (m25_zgemm_skinny): HBM-bound, 16 n^2 bytes of Z a call."""
    Z = random_matrix(n, torch.complex128)
    X = random_matrix(max(n, k), torch.complex128, seed=3)[:n, :k].contiguous()
    Y = torch.empty_like(X)
    s = torch.cuda.current_stream()
    out = []
    for r in range(reps + 1):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        check(lib().m25_zgemm_skinny(P(Z), ctypes.c_long(n), n, P(X), k, P(Y), _lib.stream_ptr()), 'm25_zgemm_skinny')
        b.record(s)
        _lib.sync_check()
        if r:
            out.append(a.elapsed_time(b))
    ms = float(np.median(out))
    return dict(n=n, k=k, ms=ms, GBps=16.0 * n * n / ms / 1e6)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--update', type=int, nargs=3, default=None, metavar=('M', 'N', 'K'))
    ap.add_argument('--solve', type=int, default=0)
    ap.add_argument('--dense', type=int, nargs=2, default=None, metavar=('N', 'K'))
    ap.add_argument('--lu', type=int, default=0)
    ap.add_argument('--single', action='store_true')
    ap.add_argument('--tf32', action='store_true')
    ap.add_argument('--reps', type=int, default=3)
    ap.add_argument('--autotune', action='store_true')
    ap.add_argument('--sizes', type=int, nargs='+', default=[2000, 5000, 10000, 20000, 40000])
    ap.add_argument('--write', action='store_true', help='write the autotuner\'s table to ' + TUNING_FILE)
    a = ap.parse_args()
    _lib.require_cuda()
    if a.autotune:
        c64 = autotune(a.sizes, single=True, reps=max(1, min(a.reps, 2)))
        c128 = autotune([n for n in a.sizes if n <= 20000], single=False, reps=1)
        print(json.dumps(dict(complex64=c64, complex128=c128)))
        if a.write:
            print('wrote', write_tuning(c64, c128))
    if a.lu:
        print(json.dumps(time_lu(a.lu, a.single, a.tf32, a.reps)))
    if a.update:
        print(json.dumps(time_update(*a.update, reps=a.reps)))
    if a.dense:
        print(json.dumps(time_dense(*a.dense, reps=a.reps)))
    if a.solve:
        print(json.dumps(time_solve(a.solve, single=a.single, reps=a.reps)))


if __name__ == '__main__':
    main()
