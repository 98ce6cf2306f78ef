"""
oracle.solve - TEST INFRASTRUCTURE ONLY: the reference's direct solve of one frequency, restated on the CPU.

  equilibrate / lu / lu_solve    fast.py:294-305, 318-320, 356-358 (symmetric diagonal scaling; LAPACK zgetrf of
                                 Z^T through SciPy, the reference's own third-party call; zgetrs with trans=1)
  gmres_batched                  fast.py:1437-1500
  Direct                         fast.py:597-605, 704-850 (fill_far + near_into_dense + via blocks, equilibrate,
                                 LU, solve: precision 'double'; 'mixed': complex64 LU refined by GMRES on the
                                 double matrix, MIXED_MAX_ITER = 30, rtol 1e-6, FRESH_STALL)
"""
import numpy as np
import scipy.linalg as sla

from . import fill_far, near_into_dense, near_coo, near_pairs, matvec_far_multi
from .green import green_tables, core_tables
from .via import fan_columns, via_blocks

MIXED_MAX_ITER = 30
FRESH_STALL = (4, 0.1)


def equilibrate(Z, dsc=None):
    if dsc is None:
        dsc = 1.0 / np.sqrt(np.abs(np.diagonal(Z)).astype(float) + 1e-300)
    dr = dsc.astype(Z.real.dtype)
    Z *= dr[:, None]
    Z *= dr[None, :]
    return dsc


def lu(Z):
    return sla.lu_factor(Z.T, overwrite_a=True, check_finite=False)


def lu_solve(f, R):
    return sla.lu_solve(f, R.astype(f[0].dtype), trans=1, check_finite=False).astype(complex)


def gmres_batched(A, B, M=None, x0=None, rtol=1e-6, restart=30, maxiter=10, stall=None):
    B = np.asarray(B, complex)
    N, k = B.shape
    X = np.zeros((N, k), complex) if x0 is None else np.array(x0, complex)
    M = M or (lambda R: R)
    bn = np.linalg.norm(B, axis=0)
    bn[bn == 0] = 1.0
    iters, act = np.zeros(k, int), np.arange(k)
    for _ in range(maxiter):
        R = B[:, act] - (A(X[:, act]) if np.any(X[:, act]) else 0)
        beta = np.linalg.norm(R, axis=0)
        done = beta <= rtol * bn[act]
        act, R, beta = act[~done], R[:, ~done], beta[~done]
        if not len(act):
            break
        ka = len(act)
        V, Zk = np.zeros((restart + 1, N, ka), complex), np.zeros((restart, N, ka), complex)
        H, g = np.zeros((restart + 1, restart, ka), complex), np.zeros((restart + 1, ka), complex)
        cs, sn = np.zeros((restart, ka), complex), np.zeros((restart, ka), complex)
        g[0], V[0] = beta, R / beta
        live, last, stalled = np.ones(ka, bool), np.full(ka, restart - 1), False
        for j in range(restart):
            Zk[j] = M(V[j])
            Wv = A(Zk[j])
            for i in range(j + 1):
                H[i, j] = hij = np.einsum('nk,nk->k', V[i].conj(), Wv)
                Wv = Wv - V[i] * hij
            H[j + 1, j] = hn = np.linalg.norm(Wv, axis=0)
            V[j + 1] = Wv / np.where(hn > 0, hn, 1)
            for i in range(j):
                H[i, j], H[i + 1, j] = (cs[i] * H[i, j] + sn[i] * H[i + 1, j],
                                        -np.conj(sn[i]) * H[i, j] + np.conj(cs[i]) * H[i + 1, j])
            den = np.sqrt(np.abs(H[j, j]) ** 2 + np.abs(H[j + 1, j]) ** 2)
            den[den == 0] = 1.0
            cs[j], sn[j] = H[j, j].conj() / den, H[j + 1, j].conj() / den
            H[j, j], H[j + 1, j] = cs[j] * H[j, j] + sn[j] * H[j + 1, j], 0
            g[j + 1], g[j] = -np.conj(sn[j]) * g[j], cs[j] * g[j]
            iters[act[live]] += 1
            conv = live & (np.abs(g[j + 1]) <= rtol * bn[act])
            last[conv] = j
            live &= ~conv
            if not live.any():
                break
            if stall is not None and j + 1 >= stall[0] and (np.abs(g[j + 1])[live] > stall[1] * bn[act][live]).any():
                last[live], stalled = j, True
                break
        for c in range(ka):
            m = last[c] + 1
            y = np.linalg.solve(np.triu(H[:m, :m, c]), g[:m, c]) if m else np.zeros(0)
            X[:, act[c]] += Zk[:m, :, c].T @ y
        if stalled:
            break
    return X, iters.tolist()


class Direct:
    """The reference's direct solver for one board (FastOperator with the compiled core), on the CPU."""

    def __init__(self, geo):
        self.geo = geo
        self.nP, self.nQ = near_pairs(geo.g['cent'], geo.tri_size, geo.tri_z, geo.near_fac)
        self.nP32, self.nQ32 = self.nP.astype(np.int32), self.nQ.astype(np.int32)
        self.q = dict(geo.q, stat=np.zeros((len(self.nP), 12)), stat_ready=False)

    def setup(self, f):
        self.f, self.w = f, 2 * np.pi * f
        self.tables = green_tables(self.geo, f)
        self.tb = core_tables(self.geo, self.tables)

    def impedance(self, f, dtype=np.complex128):
        """Z (N x N) as solve_direct assembles it (fast.py:770-790)."""
        geo = self.geo
        self.setup(f)
        Ne, N = geo.Ne, geo.N
        Z = np.zeros((N, N), dtype)
        fill_far(Z, geo.g, self.tb, self.w)
        self.qcorr = near_into_dense(Z, geo.g, self.tb, self.q, self.nP32, self.nQ32, self.w)
        self.q['stat_ready'] = True
        if geo.Nv:
            QF = fan_columns(geo, geo.g, self.tb, self.nP, self.nQ, self.qcorr)
            self.B, self.C, self.vk = via_blocks(geo, f, QF)
            Z[:Ne, Ne:], Z[Ne:, :Ne], Z[Ne:, Ne:] = self.B, self.B.T, self.C
        return Z

    def matvec_exact(self, X):
        """fast.py:571-593: Z X in double without Z (far triangle-aggregated, near COO, via blocks)."""
        geo = self.geo
        Ne = geo.Ne
        Xe = np.ascontiguousarray(X[:Ne])
        far = matvec_far_multi(Xe, geo.g, self.tb, self.w)
        near = np.zeros_like(far)
        ok = self._ri >= 0
        np.add.at(near, self._ri[ok], self._vv[ok, None] * Xe[self._ci[ok]])
        Y = np.empty(X.shape, complex)
        Y[:Ne] = far + near
        if geo.Nv:
            Y[:Ne] += self.B @ X[Ne:]
            Y[Ne:] = self.B.T @ X[:Ne] + self.C @ X[Ne:]
        return Y

    def solve(self, f, E=None, precision='double'):
        """Currents for excitation E (default: the ports'): (X, info)."""
        geo = self.geo
        E = geo.excitation() if E is None else E
        Z = self.impedance(f)
        dsc = 1.0 / np.sqrt(np.abs(np.diagonal(Z)).astype(float) + 1e-300)
        if precision == 'double':
            equilibrate(Z, dsc)
            F = lu(Z)
            X = dsc[:, None] * lu_solve(F, dsc[:, None] * E)
            return X, dict(iters=[])
        # mixed, the matrix-free double operator as the refinement's (fast.py:797-830)
        self._ri, self._ci, self._vv, _ = near_coo(geo.g, self.tb, self.q, self.nP32, self.nQ32, self.w)
        Zs = Z.copy()
        equilibrate(Zs, dsc)
        F = lu(Zs.astype(np.complex64))
        B = dsc[:, None] * E
        A = lambda V: dsc[:, None] * self.matvec_exact(dsc[:, None] * V)
        Y, it = gmres_batched(A, B, M=lambda R: lu_solve(F, R), rtol=1e-6, restart=MIXED_MAX_ITER, maxiter=1,
                              stall=FRESH_STALL)
        return dsc[:, None] * Y, dict(iters=it)

    def sparams(self, f, precision='double'):
        X, info = self.solve(f, precision=precision)
        return self.geo.sparams_from_currents(X), X, info


MIXED_RETRY = 1.25        # fast.py:252-253
REUSE_ITER = (8, 60)      # fast.py:260
REUSE_KEEP = 4            # fast.py:262


class KeptSweep:
    """The reference's CPU mixed path at sizes where a double Z fits in host memory (fast.py:704-850 with no GPU:
    `dense_kept`, then _solve_kept, fast.py:996-1084): Z filled in double (the compiled core's fill_far and
    near_into_dense, the via blocks), equilibrated; batched GMRES on the dense double Z (A = Z @ V) preconditioned
    by the complex64 LU (LAPACK cgetrf through SciPy) kept from the nearest frequency within the learnt reach
    (fast.py:974-994), capped at what a fresh one costs; else a fresh complex64 LU of Z, kept (up to keep_max);
    else the double LU of the same Z, and double up to MIXED_RETRY x f (fast.py:740-744, 1075-1084).
    core: the reference's compiled core (oracle/_ref) or this package's C restatement; same names either way."""

    def __init__(self, geo, core=None, keep_max=REUSE_KEEP, mixed_tol=1e-6):
        self.geo = geo
        self.core = core
        self.direct = Direct(geo)
        self.kept, self.reach, self.t_iter, self.mixed_failed = [], float(np.log(2.0)), None, 0.0
        self.keep_max, self.mixed_tol = keep_max, mixed_tol
        self.iters, self.last_path, self.timings = [], None, {}

    def _tick(self, name, t0):
        import time
        self.timings[name] = self.timings.get(name, 0.0) + time.perf_counter() - t0
        return time.perf_counter()

    def impedance(self, f):
        """Z at f as the reference's dense path builds it (fast.py:770-790), the compiled core where given."""
        import time
        d, geo = self.direct, self.geo
        t = time.perf_counter()
        d.setup(f)
        t = self._tick('tables', t)
        Z = np.zeros((geo.N, geo.N), complex)
        c = self.core
        (c.fill_far if c is not None else fill_far)(Z, geo.g, d.tb, d.w)
        t = self._tick('fill_far', t)
        d.qcorr = (c.near_into_dense if c is not None else near_into_dense)(Z, geo.g, d.tb, d.q, d.nP32, d.nQ32, d.w)
        d.q['stat_ready'] = True
        t = self._tick('near', t)
        if geo.Nv:
            QF = fan_columns(geo, geo.g, d.tb, d.nP, d.nQ, d.qcorr)
            d.B, d.C, d.vk = via_blocks(geo, f, QF)
            Ne = geo.Ne
            Z[:Ne, Ne:], Z[Ne:, :Ne], Z[Ne:, Ne:] = d.B, d.B.T, d.C
        self._tick('vias', t)
        return Z

    def _reusable(self, f):
        if not self.kept:
            return None
        k = min(self.kept, key=lambda k: abs(np.log(f / k[0])))
        return k if abs(np.log(f / k[0])) <= self.reach else None

    def _drop_kept(self):
        lf = np.log([k[0] for k in self.kept])
        gap = [min((abs(lf[i] - y) for j, y in enumerate(lf) if j != i), default=0.0) for i in range(len(lf))]
        del self.kept[int(np.argmin(gap))]

    def _refine(self, A, B, M, restart):
        Y, self.iters = gmres_batched(A, B, M=M, rtol=self.mixed_tol, restart=restart, maxiter=1)
        rel = np.linalg.norm(B - A(Y), axis=0) / np.maximum(np.linalg.norm(B, axis=0), 1e-300)
        return Y, bool((rel <= 100 * self.mixed_tol).all()), float(rel.max())

    def solve(self, f, E=None, precision='mixed'):
        """Currents at f for the excitation E (default: the ports'); precision 'mixed' (the reference's default
        above 3,500 unknowns, sim.py:61) or 'double'."""
        return self.solve_z(f, self.impedance(f), E, precision)

    def solve_z(self, f, Z, E=None, precision='mixed'):
        """solve() with Z at f already built (self.impedance(f)); Z is equilibrated and overwritten."""
        import time
        geo = self.geo
        E = geo.excitation() if E is None else E
        t = time.perf_counter()
        dsc = 1.0 / np.sqrt(np.abs(np.diagonal(Z)).astype(float) + 1e-300)
        equilibrate(Z, dsc)
        B = dsc[:, None] * E
        t = self._tick('equilibrate', t)
        if precision == 'mixed' and f <= MIXED_RETRY * self.mixed_failed:
            precision = 'double'
        if precision == 'double':
            F = lu(Z)
            t = self._tick('lu', t)
            X = dsc[:, None] * lu_solve(F, B)
            self._tick('solve', t)
            self.last_path = 'double'
            return X
        A = lambda V: Z @ V
        k = self._reusable(f)
        if k is not None:
            f0, F0, d0, t_fresh = k
            r = (d0 / dsc)[:, None]
            cap = int(np.clip(0.8 * t_fresh / max(self.t_iter or 1e-3, 1e-6), *REUSE_ITER))
            t1 = time.perf_counter()
            Y, ok, rel = self._refine(A, B, lambda R: r * lu_solve(F0, r * R), cap)
            self.t_iter = (time.perf_counter() - t1) / max(1, max(self.iters, default=1))
            d = abs(np.log(f / f0))
            if ok and max(self.iters) <= cap // 2:
                self.reach = max(self.reach, 1.25 * d)
            elif not ok:
                self.reach = min(self.reach, 0.8 * d)
            t = self._tick('refine', t)
            if ok:
                self.last_path = 'reused'
                return dsc[:, None] * Y
        t0 = time.perf_counter()
        F = lu(Z.astype(np.complex64))
        t = self._tick('lu', t)
        t1 = time.perf_counter()
        Y, ok, rel = self._refine(A, B, lambda R: lu_solve(F, R), MIXED_MAX_ITER)
        self.t_iter = (time.perf_counter() - t1) / max(1, max(self.iters, default=1))
        t = self._tick('refine', t)
        if ok:
            self.kept.append((f, F, dsc, time.perf_counter() - t0))
            while len(self.kept) > self.keep_max:
                self._drop_kept()
            self.last_path = 'fresh'
            return dsc[:, None] * Y
        del F
        self.mixed_failed = max(self.mixed_failed, f)
        self.last_path = 'double (after mixed)'
        X = dsc[:, None] * lu_solve(lu(Z), B)
        self._tick('lu', t)
        return X
