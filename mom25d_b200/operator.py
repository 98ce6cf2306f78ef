"""
mom25d_b200.operator - the direct solver of one board on the GPU: the drop-in for the reference's
FastOperator.solve_direct (mom25d fast.py:704-850) behind the same call, solve_direct(f, E, block, precision).

  precision='double'  complex128 Green tables, fill, near correction and via border into a device Z; symmetric
                      equilibration; complex128 LU with partial pivoting; the triangular solves. Matches the
                      reference's complex128 fill and LAPACK solve.
  precision='mixed'   where the device holds a double Z and complex64 copies (24 N^2 bytes, the reference's hybrid
                      path, fast.py:996-1084 _solve_kept): Z filled in double and equilibrated; GMRES with the dense
                      double Z (one HBM-bound product a step) preconditioned by a complex64 LU kept from a nearby
                      frequency (up to KEEP_HBM of them, reach learnt as the reference does), else by a fresh
                      complex64 LU of Z's copy (trailing updates 3xTF32 on the tensor cores when tf32=True), kept;
                      where that does not converge, the double LU of the same Z (no second fill), and double up to
                      MIXED_RETRY x f.
                      Otherwise (memory): complex64 fill from complex64 tables, the near field's double-precision
                      triplets added; complex64 LU; refined by batched GMRES (fast.py:1437-1500) on the EXACT double-
                      precision operator applied without a matrix: the triangle-aggregated far field
                      (matvec_far_multi), the near field's triplets and the via border (fast.py:571-593).
                      Either way the refinement's residuals and corrections are double precision.

Every step runs in libmom25d_b200 kernels; the host runs the GMRES recurrences on k x restart scalars.
"""
import ctypes
import time

import numpy as np
import torch

from . import _lib
from ._lib import P, check, lib, stream_ptr
from .device import DeviceGeometry, DeviceTables, DeviceVias

c_int, c_long, c_double = ctypes.c_int, ctypes.c_long, ctypes.c_double
MIXED_MAX_ITER = 30          # fast.py:255
FRESH_STALL = (4, 0.1)       # fast.py:256
MIXED_RTOL = 1e-6            # fast.py:366 (FastOperator.mixed_tol)
PREDICT_AFTER = 6            # iterations after which a fresh factor's refinement may be given up as hopeless (gmres_batched)
MIXED_RETRY = 1.25           # fast.py:252-254: after a mixed failure at f, double up to this x f
REUSE_ITER = (8, 60)         # fast.py:260: the iterations a reused LU may take (its cap, from the cost of a fresh one)
REUSE_KEEP = 4               # fast.py:262: complex64 LUs kept at most (the reference's cap, set for host memory)
KEEP_HBM = (16, 0.4)         # on the GPU: up to 16, in at most 40% of the device's memory (a complex64 LU of the
                             # routed board, N = 18,788, is 2.8 GB). More kept factors leave a nearer one for each
                             # frequency of a sweep: a reuse at 1.16x the kept frequency takes ~10 GMRES steps
                             # (~100 ms) where a fresh factor takes ~215 ms (measured on the routed board)
REUSE_GIVE_UP = (10, 0.05)   # a reused factor's GMRES ends from step 10 where a residual is still above 5% of |b| (a
                             # fresh LU follows). Rules that projected the rate of the last few steps to the cap were
                             # measured and dropped: GMRES plateaus and then speeds up, and they cut off attempts that
                             # converged in 25 steps
FRESH_STAGNATION = (10, 0.5)  # a fresh factor's GMRES ends at step 10 where a residual has not halved since step 1
                             # (measured on the routed board: at 0.5 GHz it stays at 2e-3 for all 30 steps; at 0.67 GHz
                             # it is 5x lower by step 10 and converges at 27)
REACH_WINDOW = float(0.5 * np.log(2.0))  # _reach_at: the attempts within half an octave of f set its reach (an
                             # octave let the 4.07 GHz failure of the routed board stop the reuses at 2.24 GHz)
DOUBLE_REACH = float(np.log(1.6))  # |ln f / f0| within which the kept double factor preconditions a double solve
DOUBLE_UP = 1.6              # after a complex64 failure at f0, the frequencies up to this x f0 with the kept double factor
                             # within reach go to it directly, past the reference's MIXED_RETRY: a complex64 factor is
                             # as marginal there (its backward error times the condition of Z near 1: measured on the
                             # routed board, a fresh complex64 LU at 0.67 and 0.78 GHz after 0.5 GHz failed converged or
                             # stalled with rounding noise, a 990 ms step when it stalls) and the kept double factor
                             # converges in ~5 GMRES steps


SMALL = 1e-300


class SolveFailed(RuntimeError):
    """The mixed-precision refinement did not converge (the caller redoes the frequency in double)."""


class DirectSolver:
    """One board's device-resident direct solver (meshes, pairs, tables and factors stay on the GPU)."""

    def __init__(self, geo, stream=None, tf32=False, log=None, keep=None):
        """keep: complex64 LUs kept for reuse at most (None: KEEP_HBM, memory allowing; REUSE_KEEP is the
        reference's own cap)."""
        self.geo, self.stream = geo, stream
        self.keep = keep
        self.dg = DeviceGeometry(geo, stream)
        self.tf32 = tf32
        self.log = log if log is not None else []
        self.timings = {}
        self.iters = []
        self._work = {}
        self.kept = []                     # (f, factor record, dsc, seconds the fresh solve took): _solve_kept
        self.reach = float(np.log(2.0))    # fast.py:862: |ln(f / f0)| within which a kept LU is tried, at first
        self.reach_log = []                # reuse attempts (f, |ln f / f0|, converged, iterations, cap): _reach_at
        self.t_iter = None
        self.mixed_failed = 0.0
        self.reuse = True
        self.hybrid = 'auto'               # 'auto' (when the double Z fits), True, False
        self.last_path = None
        self.last_lu_ms = self.last_lu_c64_ms = None
        self.attempts = []                 # reused-LU attempts: (f, f0, cap, iterations, converged, residual)
        self.extras = None                 # extras.ExtraBlocks: lumped elements, conductor loss (fast.py:628-641)
        self.kept64 = None                 # (f, factor record, dsc, seconds): the last double LU made next to a
                                           # complex64 failure, preconditioning the double solves near it
        self.t_iter64 = None

    # ---- buffers kept across frequencies ---------------------------------------------------------------------------
    def _buf(self, name, shape, dtype):
        t = self._work.get(name)
        if t is None or t.shape != tuple(shape) or t.dtype != dtype:
            t = torch.empty(shape, dtype=dtype, device='cuda')
            self._work[name] = t
        return t

    def _getrf_work(self, n, single):
        nbytes = int(lib().m25_getrf_workspace(c_int(n), c_int(1 if single else 0)))
        return self._buf('getrf_work_%d' % single, (nbytes,), torch.uint8)

    # ---- device memory ------------------------------------------------------------------------------------------------
    def release(self):
        """Drops every per-frequency buffer (Z, its complex64 copies and factors, kept LUs, workspaces, Krylov
        bases, tables); what stays is the per-board state (resident_bytes). The memory goes back to torch's
        caching allocator."""
        self._work.clear()
        self.kept, self.kept64 = [], None
        for name in ('aux', 'tabs', 'vias', 'ri', 'ci', 'vv', 'Bv', 'Cv'):
            if hasattr(self, name):
                delattr(self, name)
        if self.extras is not None:
            self.extras._vals, self.extras._vals_f = None, None

    def resident_bytes(self):
        """Device bytes the board's state holds between requests: mesh, quadrature, near pairs and their kept
        analytic moments, the via index lists."""
        seen, total = set(), 0
        for t in list(self.dg.__dict__.values()) + list(self.dg.t.values()) + list(self.dg.tq.values()) + \
                [g[k] for g in getattr(self.dg, 'groups', []) for k in ('m', 'n', 'dd')]:
            if torch.is_tensor(t) and t.is_cuda and t.data_ptr() not in seen:
                seen.add(t.data_ptr())
                total += t.numel() * t.element_size()
        return total

    def held_bytes(self):
        """Device bytes this solver holds now beyond its resident state (per-frequency buffers and kept factors)."""
        total = sum(t.numel() * t.element_size() for t in self._work.values())
        total += sum(k[1]['bytes'] for k in self.kept)
        if self.kept64 is not None:
            total += self.kept64[1]['Z'].numel() * 16 + self.kept64[1]['aux'].numel()
        return total

    @property
    def s(self):
        return stream_ptr(self.stream)

    # ---- phase timings: CUDA events on the solver's stream (no host synchronisation on the path) ------------------
    def _mark(self):
        e = torch.cuda.Event(enable_timing=True)
        e.record(self.stream if self.stream is not None else torch.cuda.current_stream())
        return e

    def _t(self, name, e0):
        """The device time from event e0 (self._mark()) to now is added to phase `name`."""
        self._pending.append((name, e0, self._mark()))

    @property
    def timings(self):
        """Seconds per phase so far (tables, fill, vias, lu, refine, refine_matvec, refine_precond, solve)."""
        if self._pending:
            self._pending[-1][2].synchronize()
            for name, a, b in self._pending:
                self._timings[name] = self._timings.get(name, 0.0) + a.elapsed_time(b) / 1000.0
            self._pending = []
        return self._timings

    @timings.setter
    def timings(self, value):
        self._pending, self._timings = [], dict(value)

    # ---- tables and fill -----------------------------------------------------------------------------------------
    def setup(self, f, single=False):
        self.f, self.w = f, 2 * np.pi * f
        self.tabs = DeviceTables(self.dg, f, single=single, stream=self.stream)
        self.vias = DeviceVias(self.dg, self.tabs, self.stream)

    def impedance(self, f, precision='double', far=None):
        """Z at f on the device: complex128 (double) or complex64 (mixed). far: a complex128 N x N tensor whose far
        part at f is already filled (m25_fill_far_multi with this board's tables at f, the batched sweep): the near
        field, the via border and the extra blocks are added into it, and it is returned."""
        geo, dg = self.geo, self.dg
        N, Ne = geo.N, geo.Ne
        single = precision == 'mixed'
        t0 = self._mark()
        self.setup(f, single=single)
        self._t('tables', t0)
        tb, s = self.tabs, self.s
        t0 = self._mark()
        qcorr = self._buf('qcorr', (max(1, dg.npairs),), torch.complex128)
        if not single:
            if far is not None:
                Z = far
            else:
                Z = self._buf('Z', (N, N), torch.complex128)
                check(lib().m25_fill_far(P(Z), c_long(N), c_int(0), ctypes.byref(dg.mesh), ctypes.byref(tb.tables),
                                         None, c_double(self.w), s), 'm25_fill_far')
            check(lib().m25_near(c_int(0), P(Z), c_long(N), c_int(0), None, None, None, P(qcorr), P(dg.stat),
                                 c_int(int(dg.stat_ready)), ctypes.byref(dg.mesh), ctypes.byref(tb.tables),
                                 ctypes.byref(dg.quad), P(dg.nP), P(dg.nQ), c_long(dg.npairs), c_double(self.w), s),
                  'm25_near')
            dg.stat_ready = True
            self._t('fill', t0)
            t0 = self._mark()
            self.vias.assemble(Z, N, qcorr)
            self._t('vias', t0)
            if self.extras is not None:                   # lumped elements, conductor loss (fast.py:628-641)
                self.extras.add(Z, f, self.stream)
            return Z
        Z = self._buf('Z64', (N, N), torch.complex64)
        check(lib().m25_fill_far(P(Z), c_long(N), c_int(1), ctypes.byref(dg.mesh), None, ctypes.byref(tb.tables32),
                                 c_double(self.w), s), 'm25_fill_far')
        nnz = 9 * dg.npairs
        self.ri = self._buf('ri', (max(1, nnz),), torch.int32)
        self.ci = self._buf('ci', (max(1, nnz),), torch.int32)
        self.vv = self._buf('vv', (max(1, nnz),), torch.complex128)
        check(lib().m25_near(c_int(2), None, c_long(0), c_int(0), P(self.ri), P(self.ci), P(self.vv), P(qcorr),
                             P(dg.stat), c_int(int(dg.stat_ready)), ctypes.byref(dg.mesh), ctypes.byref(tb.tables),
                             ctypes.byref(dg.quad), P(dg.nP), P(dg.nQ), c_long(dg.npairs), c_double(self.w), s),
              'm25_near')
        dg.stat_ready = True
        check(lib().m25_coo_add_c64(P(self.ri), P(self.ci), P(self.vv), c_long(nnz), P(Z), c_long(N), s),
              'm25_coo_add_c64')
        self.Bv = self._buf('Bv', (max(1, Ne * geo.Nv),), torch.complex128)
        self.Cv = self._buf('Cv', (max(1, geo.Nv * geo.Nv),), torch.complex128)
        self._t('fill', t0)
        t0 = self._mark()
        self.vias.assemble(None, N, qcorr, Z64=Z, B=self.Bv, C=self.Cv)
        self._t('vias', t0)
        if self.extras is not None:
            self.extras.add(Z, f, self.stream)
        return Z

    # ---- the exact double-precision operator (fast.py:571-593) --------------------------------------------------------
    def matvec_exact(self, X):
        """Z X in double precision without Z: X (N x k) complex128 device tensor -> new tensor."""
        geo, dg, s = self.geo, self.dg, self.s
        N, Ne, k = geo.N, geo.Ne, X.shape[1]
        X = X.contiguous()
        Y = torch.empty_like(X)
        Xe = X[:Ne].contiguous()
        work = self._buf('mv_work', (6 * geo.Nt * k,), torch.complex128)
        Ye = torch.empty((Ne, k), dtype=torch.complex128, device='cuda')
        check(lib().m25_matvec_far_multi(P(Xe), c_int(k), P(Ye), P(work), ctypes.byref(dg.mesh),
                                         ctypes.byref(self.tabs.tables), c_double(self.w), s), 'm25_matvec_far_multi')
        check(lib().m25_near_spmm_rows(ctypes.byref(dg.mesh), P(dg.off), P(dg.nQ), P(self.vv), P(Xe), c_int(k), P(Ye),
                                       s), 'm25_near_spmm_rows')
        Y[:Ne] = Ye
        if geo.Nv:
            check(lib().m25_border_mv(P(self.Bv), P(self.Cv), c_int(Ne), c_int(geo.Nv), P(X), c_int(k), P(Y), s),
                  'm25_border_mv')
        if self.extras is not None:                       # + S X, the lumped elements and conductor loss
            self.extras.apply(X, Y, self.f, self.stream)
        return Y

    # ---- device vector helpers ------------------------------------------------------------------------------------------
    def _dotc(self, V, W):
        k = V.shape[1]
        out = self._buf('dot', (k,), torch.complex128)
        check(lib().m25_dotc_cols(P(V), P(W), c_long(V.shape[0]), c_int(k), P(out), self.s), 'm25_dotc_cols')
        return out.cpu().numpy().copy()

    def _axpy_multi(self, W, Vall, nv, h):
        """W -= sum_i V_i h[i] (per column)."""
        N, k = W.shape
        h_d = _lib.dev(np.ascontiguousarray(h, complex))
        check(lib().m25_axpy_multi(P(W), P(Vall), c_int(nv), c_long(N), c_int(k), P(h_d), self.s), 'm25_axpy_multi')

    def _scale(self, X, s_cols=None, rows=None, out=None):
        Y = torch.empty_like(X) if out is None else out
        sc = None if s_cols is None else _lib.dev(np.asarray(s_cols, complex))
        check(lib().m25_scale_cols(P(Y), P(X), P(sc), P(rows), c_long(X.shape[0]), c_int(X.shape[1]), self.s),
              'm25_scale_cols')
        return Y

    # ---- solves -------------------------------------------------------------------------------------------------------
    def _factor(self, Z, single):
        """LU of Z (double, or complex64 with single=True) in place, and the prepared solve data; the pivots."""
        N = self.geo.N
        ipiv = self._buf('ipiv', (N,), torch.int32)
        work = self._getrf_work(N, single)
        a = self._mark()
        check(lib().m25_getrf(P(Z), c_long(N), c_int(N), P(ipiv), c_int(int(single)),
                              c_int(int(single and self.tf32)), P(work), ctypes.c_size_t(work.numel()), self.s),
              'm25_getrf')
        b = self._mark()
        _lib.sync_check(self.stream, 'm25_getrf')
        self.last_lu_ms = a.elapsed_time(b)                # the factorisation alone, on its stream
        self._pending.append(('lu', a, b))
        # the solves' diagonal-block inverses and row permutation, once per factor
        nbytes = int(lib().m25_getrs_aux_bytes(c_int(N), c_int(int(single))))
        self.aux = self._buf('getrs_aux_%d' % single, (nbytes,), torch.uint8)
        check(lib().m25_getrs_prepare(P(Z), c_long(N), c_int(N), P(ipiv), c_int(int(single)), P(self.aux),
                                      ctypes.c_size_t(nbytes), self.s), 'm25_getrs_prepare')
        return ipiv

    def _lu_solve(self, Z, ipiv, R, single):
        """Z^-1 R with the factor (lu_solve(..., trans=1)), R complex128 (N x k) -> complex128."""
        N, k = R.shape
        if single:
            return self._solve_c64(dict(Z=Z, aux=self.aux), R)
        X = R.clone()
        check(lib().m25_getrs_aux(P(Z), c_long(N), c_int(N), c_int(0), P(self.aux), P(X), c_int(k), self.s),
              'm25_getrs_aux')
        return X

    def solve_direct(self, f, E, block=1024, precision='double', far=None):
        """Currents for the excitation columns E (N x k, host or device): a complex128 device tensor. far: Z with its
        far part at f already filled (impedance), used in place of a new fill by the mixed path with a resident
        double Z (the batched sweep)."""
        geo = self.geo
        N = geo.N
        E = torch.as_tensor(np.asarray(E) if not torch.is_tensor(E) else E, dtype=torch.complex128).to('cuda')
        E = E.reshape(N, -1).contiguous()
        self.iters = []
        self.last_lu_ms = self.last_lu_c64_ms = None
        if precision == 'mixed' and self._double_band(f):
            precision = 'double'                          # fast.py:740: near a failure, double
            if self._hybrid_fits():
                return self._solve_double_near(f, E)
        if precision == 'mixed' and (far is not None or self._hybrid_fits()):
            return self._solve_kept(f, E, far)
        self.last_path = precision
        single = precision == 'mixed'
        Z = self.impedance(f, precision)
        dsc = self._buf('dsc', (N,), torch.float64)
        if single:
            check(lib().m25_equilibrate_c64(P(Z), c_long(N), c_long(N), P(dsc), self.s), 'm25_equilibrate_c64')
        else:
            check(lib().m25_equilibrate(P(Z), c_long(N), c_long(N), None, P(dsc), None, self.s), 'm25_equilibrate')
        ipiv = self._factor(Z, single)
        t0 = self._mark()
        B = self._scale(E, rows=dsc)
        if not single:
            Y = self._lu_solve(Z, ipiv, B, False)
            X = self._scale(Y, rows=dsc)
            self._t('solve', t0)
            return X
        A = lambda V: self._timed('refine_matvec', lambda: self._scale(self.matvec_exact(self._scale(V, rows=dsc)),
                                                                       rows=dsc))
        M = lambda R: self._timed('refine_precond', lambda: self._lu_solve(Z, ipiv, R, True))
        Y, ok, rel = self.refine(A, B, M, MIXED_MAX_ITER, FRESH_STALL)
        self._t('refine', t0)
        if not ok:
            raise SolveFailed(f"mixed precision did not converge at {f / 1e9:.4g} GHz (residual {rel:.1e})")
        return self._scale(Y, rows=dsc)

    # ---- mixed precision with a resident double Z and kept complex64 LUs (fast.py:996-1118) ------------------------
    def _hybrid_fits(self):
        """Room for the double Z, a complex64 copy to factor and the workspaces (fast.py:720-728, on the device)."""
        if self.hybrid != 'auto':
            return bool(self.hybrid)
        N = self.geo.N
        free, _ = torch.cuda.mem_get_info()
        held = sum(t.numel() * t.element_size() for t in self._work.values())
        return 24.0 * N * N + 1e9 <= 0.8 * (free + held)

    def _keep_max(self):
        """LUs that may stay resident (fast.py:959-960, memory allowing, 8 N^2 bytes each): the cap is keep, else
        KEEP_HBM's count within its share of the device's memory."""
        if not self.reuse:
            return 0
        N = self.geo.N
        free, total = torch.cuda.mem_get_info()
        kept = sum(k[1]['bytes'] for k in self.kept)
        cap = self.keep if self.keep is not None else min(KEEP_HBM[0], int(KEEP_HBM[1] * total // (8.0 * N * N)))
        return int(min(cap, (0.9 * (free + kept) - 0.4e9) // (8.0 * N * N)))

    def _double_band(self, f):
        """Whether a mixed request at f is solved in double: up to MIXED_RETRY x the highest complex64 failure (the
        reference's rule, fast.py:740), and up to DOUBLE_UP x it where the kept double factor is within
        DOUBLE_REACH of f."""
        if f <= MIXED_RETRY * self.mixed_failed:
            return True
        return (self.kept64 is not None and f <= DOUBLE_UP * self.mixed_failed and
                abs(np.log(f / self.kept64[0])) <= DOUBLE_REACH)

    def forget(self):
        """A new sweep: no kept factors, nothing learnt."""
        self.kept, self.reach_log, self.t_iter, self.mixed_failed = [], [], None, 0.0
        self.kept64, self.t_iter64 = None, None
        self.reach = float(np.log(2.0))

    def _reusable(self, f):
        """fast.py:974-980: the kept LU nearest in frequency, if within the reach at f."""
        if not self.reuse or not self.kept:
            return None
        k = min(self.kept, key=lambda k: abs(np.log(f / k[0])))
        return k if abs(np.log(f / k[0])) <= self._reach_at(f) else None

    def _reach_at(self, f):
        """The reach at f: the reference's rule (fast.py:989-994: a quick success widens it to 1.25 d, a failure
        narrows it to 0.8 d) replayed over the attempts within half an octave of f (REACH_WINDOW), in the order
        they were made. The
        reference learns one reach for the whole band; how fast Z moves with f depends on where in the band f is
        (measured on the routed board: reuses converge at 1.57x the kept frequency around 1-3 GHz and fail at
        1.16x above 5 GHz), so a failure at 6 GHz no longer stops the reuses at 2 GHz."""
        r = self.reach
        for fa, d, ok, iters, cap in self.reach_log:
            if abs(np.log(f / fa)) > REACH_WINDOW:
                continue
            if ok and iters <= cap // 2:
                r = max(r, 1.25 * d)
            elif not ok:
                r = min(r, 0.8 * d)
        return r

    def _drop_kept(self):
        """fast.py:982-987: drop the kept LU nearest another kept one."""
        lf = np.log([k[0] for k in self.kept])
        gap = [min((abs(lf[i] - y) for j, y in enumerate(lf) if j != i), default=0.0) for i in range(len(lf))]
        del self.kept[int(np.argmin(gap))]

    def _reach_learn(self, f, d, ok, iters, cap):
        """fast.py:989-994: an attempt at f with a factor kept at |ln f / f0| = d, for _reach_at."""
        self.reach_log.append((f, d, bool(ok), max(iters, default=0), cap))

    def _factor_c64(self, Z64):
        """A complex64 LU of its own (kept across frequencies): the factor in Z64's memory, pivots, the solves'
        prepared diagonal-block inverses."""
        N = self.geo.N
        rec = dict(Z=Z64, ipiv=torch.empty(N, dtype=torch.int32, device='cuda'))
        work = self._getrf_work(N, True)
        a = self._mark()
        check(lib().m25_getrf(P(Z64), c_long(N), c_int(N), P(rec['ipiv']), c_int(1), c_int(int(self.tf32)), P(work),
                              ctypes.c_size_t(work.numel()), self.s), 'm25_getrf')
        b = self._mark()
        _lib.sync_check(self.stream, 'm25_getrf')
        self.last_lu_ms = self.last_lu_c64_ms = a.elapsed_time(b)
        self._pending.append(('lu', a, b))
        nbytes = int(lib().m25_getrs_aux_bytes(c_int(N), c_int(1)))
        rec['aux'] = torch.empty(nbytes, dtype=torch.uint8, device='cuda')
        check(lib().m25_getrs_prepare(P(Z64), c_long(N), c_int(N), P(rec['ipiv']), c_int(1), P(rec['aux']),
                                      ctypes.c_size_t(nbytes), self.s), 'm25_getrs_prepare')
        rec['bytes'] = Z64.numel() * 8 + nbytes
        return rec

    def _solve_c64(self, rec, R):
        """Z^-1 R with a complex64 factor, R complex128 (N x k) -> complex128."""
        N, k = R.shape
        R64 = torch.empty((N, k), dtype=torch.complex64, device='cuda')
        check(lib().m25_convert(P(R), c_int(0), P(R64), c_long(N * k), self.s), 'm25_convert')
        check(lib().m25_getrs_aux(P(rec['Z']), c_long(N), c_int(N), c_int(1), P(rec['aux']), P(R64), c_int(k), self.s),
              'm25_getrs_aux')
        X = torch.empty((N, k), dtype=torch.complex128, device='cuda')
        check(lib().m25_convert(P(R64), c_int(1), P(X), c_long(N * k), self.s), 'm25_convert')
        return X

    def _dense(self, Z, V):
        """Z V for the resident double Z (row-major N x N) and V (N x k), k <= 16 a call."""
        N, k = V.shape
        V = V.contiguous()
        Y = torch.empty_like(V)
        for c0 in range(0, k, 16):
            c1 = min(k, c0 + 16)
            Vc = V[:, c0:c1].contiguous() if (c0, c1) != (0, k) else V
            Yc = Y if (c0, c1) == (0, k) else torch.empty_like(Vc)
            check(lib().m25_zgemm_skinny(P(Z), c_long(N), c_int(N), P(Vc), c_int(c1 - c0), P(Yc), self.s),
                  'm25_zgemm_skinny')
            if Yc is not Y:
                Y[:, c0:c1] = Yc
        return Y

    def _solve_kept(self, f, E, far=None):
        """fast.py:996-1084 on the device: returns the currents (equilibration undone)."""
        N = self.geo.N
        Z = self.impedance(f, 'double', far)
        dsc = self._buf('dsc', (N,), torch.float64)
        check(lib().m25_equilibrate(P(Z), c_long(N), c_long(N), None, P(dsc), None, self.s), 'm25_equilibrate')
        dsc = dsc.clone()
        B = self._scale(E, rows=dsc)
        A = lambda V: self._timed('refine_matvec', lambda: self._dense(Z, V))
        k = self._reusable(f)
        if k is not None:
            f0, rec, d0, t_fresh = k
            r = (d0 / dsc).contiguous()                   # Zs^-1 ~ (D0 / D) Z0s^-1 (D0 / D)
            cap = int(np.clip(0.8 * t_fresh / max(self.t_iter or 1e-3, 1e-6), *REUSE_ITER))
            M = lambda R: self._timed('refine_precond', lambda: self._scale(self._solve_c64(rec, self._scale(R, rows=r)),
                                                                              rows=r))
            e0, t = self._mark(), time.perf_counter()
            Y, ok, rel = self.refine(A, B, M, cap, give_up=REUSE_GIVE_UP)
            self._learn_t_iter((time.perf_counter() - t) / max(1, max(self.iters, default=1)))
            self._reach_learn(f, abs(np.log(f / f0)), ok, self.iters, cap)
            self.attempts.append(dict(f=f, f0=f0, cap=cap, iters=max(self.iters, default=0), ok=ok, rel=rel))
            self._t('refine', e0)
            if ok:
                self.last_path = 'reused'
                return self._scale(Y, rows=dsc)
        t_fresh0 = time.perf_counter()
        keep_max = self._keep_max()
        while self.kept and len(self.kept) >= max(1, keep_max):
            self._drop_kept()                             # room for the new factor
        Z64 = torch.empty((N, N), dtype=torch.complex64, device='cuda')
        check(lib().m25_convert(P(Z), c_int(0), P(Z64), c_long(N * N), self.s), 'm25_convert')
        rec = self._factor_c64(Z64)
        M = lambda R: self._timed('refine_precond', lambda: self._solve_c64(rec, R))
        e0, t = self._mark(), time.perf_counter()
        Y, ok, rel = self.refine(A, B, M, MIXED_MAX_ITER, FRESH_STALL, predict=False, stagnate=FRESH_STAGNATION)
        self._learn_t_iter((time.perf_counter() - t) / max(1, max(self.iters, default=1)))
        self._t('refine', e0)
        if ok:
            self.last_path = 'fresh'
            if keep_max >= 1:
                self.kept.append((f, rec, dsc, time.perf_counter() - t_fresh0))
            return self._scale(Y, rows=dsc)
        del rec, Z64
        # the double LU of the same (equilibrated) Z, and double up to MIXED_RETRY x f (fast.py:1074-1084); that LU
        # is kept to precondition the double solves near f (_solve_double_near)
        self.mixed_failed = max(self.mixed_failed, f)
        self.log.append(f"mixed precision did not converge at {f / 1e9:.4g} GHz (residual {rel:.1e}): double LU of the "
                        f"same Z, double up to {MIXED_RETRY * f / 1e9:.4g} GHz")
        self.last_path = 'double (after mixed)'
        return self._double_fresh(f, Z, dsc, B, time.perf_counter())

    def _double_fresh(self, f, Z, dsc, B, t0):
        """A double LU of the equilibrated Z (in place) and its solve; the factor is kept (self.kept64), its memory
        leaving the solver's work buffers."""
        ipiv = self._factor(Z, False)
        e0 = self._mark()
        X = self._lu_solve(Z, ipiv, B, False)
        self._t('solve', e0)
        rec = dict(Z=Z, aux=self.aux, ipiv=ipiv)
        for name in ('Z', 'getrs_aux_0', 'ipiv'):         # the next fill and factor take new buffers
            self._work.pop(name, None)
        self.kept64 = (f, rec, dsc.clone(), time.perf_counter() - t0)
        return self._scale(X, rows=dsc)

    def _solve_c128(self, rec, R):
        """Z^-1 R with a kept double factor, R complex128 (N x k)."""
        N, k = R.shape
        X = R.clone()
        check(lib().m25_getrs_aux(P(rec['Z']), c_long(N), c_int(N), c_int(0), P(rec['aux']), P(X), c_int(k), self.s),
              'm25_getrs_aux')
        return X

    def _solve_double_near(self, f, E):
        """A frequency the reference solves in double because the complex64 factor failed near it (fast.py:740):
        GMRES on the dense double Z preconditioned by the double LU kept from the failure's neighbourhood (within
        DOUBLE_REACH in |ln f / f0|, scaled by the equilibrations as kept complex64 LUs are), capped at what a
        fresh double LU costs; a fresh double LU (then kept) where there is none or it does not converge."""
        N = self.geo.N
        t0 = time.perf_counter()
        Z = self.impedance(f, 'double')
        dsc = self._buf('dsc', (N,), torch.float64)
        check(lib().m25_equilibrate(P(Z), c_long(N), c_long(N), None, P(dsc), None, self.s), 'm25_equilibrate')
        dsc = dsc.clone()
        B = self._scale(E, rows=dsc)
        k = self.kept64
        if k is not None and abs(np.log(f / k[0])) <= DOUBLE_REACH:
            f0, rec, d0, t_fresh = k
            r = (d0 / dsc).contiguous()
            cap = int(np.clip(0.8 * t_fresh / max(self.t_iter64 or 0.04, 1e-6), *REUSE_ITER))
            A = lambda V: self._timed('refine_matvec', lambda: self._dense(Z, V))
            M = lambda R: self._timed('refine_precond', lambda: self._scale(self._solve_c128(rec, self._scale(R, rows=r)),
                                                                              rows=r))
            e0, t = self._mark(), time.perf_counter()
            Y, ok, rel = self.refine(A, B, M, cap, give_up=REUSE_GIVE_UP)
            it = max(1, max(self.iters, default=1))
            self.t_iter64 = (time.perf_counter() - t) / it if self.t_iter64 is None else \
                min(self.t_iter64, (time.perf_counter() - t) / it)
            self._t('refine', e0)
            self.attempts.append(dict(f=f, f0=f0, cap=cap, iters=max(self.iters, default=0), ok=ok, rel=rel,
                                      double=True))
            if ok:
                self.last_path = 'reused double'
                return self._scale(Y, rows=dsc)
        self.last_path = 'double'
        return self._double_fresh(f, Z, dsc, B, t0)

    def _learn_t_iter(self, t):
        """The time of one refinement iteration, which sets a reused LU's cap (fast.py:1019): the smallest seen, so
        that a first solve's one-off costs (kernel loading, buffers) do not shrink the caps that follow."""
        self.t_iter = t if self.t_iter is None else min(self.t_iter, t)

    def _timed(self, name, fn):
        e = self._mark()
        out = fn()
        self._t(name, e)
        return out

    # ---- the refinement: batched right-preconditioned GMRES (fast.py:658-663, 1437-1500) -----------------------------
    def refine(self, A, B, M, restart, stall=None, predict=True, give_up=None, stagnate=None):
        """fast.py:658-663: GMRES to MIXED_RTOL, one cycle of at most `restart` iterations; (Y, converged, largest
        relative residual of B - A Y)."""
        Y, self.iters = self.gmres_batched(A, B, M, rtol=MIXED_RTOL, restart=restart, stall=stall, predict=predict,
                                           give_up=give_up, stagnate=stagnate)
        R = B - A(Y)
        rn = np.sqrt(np.abs(self._dotc(R, R)))
        bn = np.sqrt(np.abs(self._dotc(B, B)))
        rel = rn / np.maximum(bn, 1e-300)
        self.residual = rel
        return Y, bool(np.isfinite(rel).all() and (rel <= 100 * MIXED_RTOL).all()), float(rel.max())

    def gmres_batched(self, A, B, M, rtol=1e-6, restart=30, stall=None, predict=True, give_up=None, stagnate=None):
        """Right-preconditioned GMRES on A Y = B for the k columns of B at once, one cycle from Y = 0, the role of
        the reference's gmres_batched (fast.py:1437-1500) as its callers use it (maxiter 1, fast.py:1053):

        - the Krylov bases of all columns advance together: the directions Z_j = M(V_j) and A Z_j are N x k
          blocks, and m25_arnoldi_orth orthogonalises A Z_j against V_0 .. V_j (classical Gram-Schmidt applied
          twice) and normalises it into V_{j+1} on the device, leaving the Hessenberg column there;
        - the host reads that column (the one synchronisation of a step) and, for each column still iterating,
          solves the small least-squares problem min |beta e_1 - H y| by a complete QR of H, whose last
          transformed entry is the residual norm;
        - a column whose residual reaches rtol |b| stops there (its y from that step); the others go on;
        - stall = (n, x): after n steps, a column still above x |b| ends the iteration for all (the reference's
          FRESH_STALL rule, fast.py:256); with predict, after PREDICT_AFTER steps a column whose geometric rate
          so far would leave it 10x above the tolerance at the last step also ends it (the caller will solve in
          double precision: the steps that remain would be lost);
        - give_up = (n, x): from step n a column whose residual is still above x |b| ends the iteration (a
          reused factor that will not converge within its cap gives way to a fresh one sooner);
        - stagnate = (n, x): at step n a column whose residual is above x times its residual after the first step
          ends the iteration (a fresh factor too weak to precondition: the caller solves in double precision);
        - Y = sum_j Z_j y_j, one device product per step used.
        Returns (Y, iterations per column)."""
        N, k = B.shape
        bn = np.sqrt(np.abs(self._dotc(B, B)))
        bn[bn == 0] = 1.0
        V = self._buf('krylov', (restart + 1, N, k), torch.complex128)
        Zd = self._buf('krylov_z', (restart, N, k), torch.complex128)
        hcol = self._buf('hcol', (restart + 1, k), torch.complex128)
        htmp = self._buf('htmp', (restart + 1, k), torch.complex128)
        # V_0 = B / |B| per column
        self._scale(B, s_cols=1.0 / bn, out=V[0])
        H = np.zeros((k, restart + 1, restart), complex)
        rhs = np.zeros((k, restart + 1), complex)
        rhs[:, 0] = bn
        steps = np.zeros(k, int)              # steps each column takes (its y has that many entries)
        done = np.zeros(k, bool)
        res = bn.copy()
        hist = [bn.copy()]
        for j in range(restart):
            Zd[j].copy_(M(V[j]))
            W = A(Zd[j]).contiguous()
            check(lib().m25_arnoldi_orth(P(V), c_int(j), c_long(N), c_int(k), P(W), P(hcol), P(htmp), self.s),
                  'm25_arnoldi_orth')
            H[:, :j + 2, j] = hcol[:j + 2].cpu().numpy().T
            live = np.flatnonzero(~done)
            Q, _ = np.linalg.qr(H[live, :j + 2, :j + 1], mode='complete')
            g = np.einsum('cji,cj->ci', Q.conj(), rhs[live, :j + 2])
            res[live] = np.abs(g[:, j + 1])
            steps[live] = j + 1
            done[live] |= res[live] <= rtol * bn[live]
            hist.append(res.copy())
            if done.all():
                break
            act = ~done
            if give_up is not None and j + 1 >= give_up[0] and j + 1 < restart and \
                    (res[act] > give_up[1] * bn[act]).any():
                break
            if stagnate is not None and j + 1 == stagnate[0] and j + 1 < restart and \
                    (res[act] > stagnate[1] * hist[1][act]).any():
                break
            if stall is not None and j + 1 >= stall[0] and (res[act] > stall[1] * bn[act]).any():
                break
            if stall is not None and predict and j + 1 >= PREDICT_AFTER:
                rate = (res[act] / bn[act]) ** (1.0 / (j + 1))
                if (res[act] * rate ** (restart - j - 1) > 10 * rtol * bn[act]).any():
                    break
        # the largest relative residual estimate after each step (diagnostics: the bench's verbose log)
        self.res_hist = [float((h / bn).max()) for h in hist]
        # y per column from its own steps, Y = sum_j Z_j y_j
        m = int(steps.max())
        coef = np.zeros((m, k), complex)
        for c in range(k):
            s_c = steps[c]
            Q, R = np.linalg.qr(H[c, :s_c + 1, :s_c], mode='complete')
            g = Q.conj().T @ rhs[c, :s_c + 1]
            coef[:s_c, c] = np.linalg.solve(np.triu(R[:s_c, :s_c]), g[:s_c])
        Y = torch.zeros((N, k), dtype=torch.complex128, device='cuda')
        if m:
            self._axpy_multi(Y, Zd, m, -coef)
        return Y, steps.tolist()
