"""
oracle.green - TEST INFRASTRUCTURE ONLY: NumPy restatement of the reference's layered-media Green tables.

  network / voltage / spectral   multilayer.py:183-250 (the stack's transmission-line network, TE 'h' / TM 'e')
  sommerfeld_contour             via.py:36-53
  hankel                         via.py:90-108 (real part of the contour: oracle.c's glibc-j0 sum; lifted part:
                                 oracle.c's J_n series / Hankel expansion, mom25d_core.cpp:1510-1543)
  GreenTable                     multilayer.py:253-318 (singular parts taken out spectrally, CubicSpline to nfine)
  green_tables / core_tables     sim.py:736-745, fast.py:556-568 (which pairs, what they extract, the tb dict)
"""
import numpy as np
from scipy.interpolate import CubicSpline

from . import bessel_jn_complex, hankel_real

MU0 = 4e-7 * np.pi
C0 = 299792458.0
EPS0 = 1.0 / (MU0 * C0 ** 2)


def network(st, kr, w, mode):
    """multilayer.py:183-219 for a stack over a PEC ground with an open or PEC top and no planes inside."""
    k0, N = w / C0, st.N

    def y0(e):
        kz = -1j * np.sqrt(kr ** 2 - k0 ** 2 * e)
        return kz / (w * MU0) if mode == 'h' else w * EPS0 * e / kz, kz
    Y0, tn, sc = [None] * (N + 1), [None] * (N + 1), [None] * (N + 1)
    for j in range(1, N + 1):
        Y0[j], kz = y0(st.eps(j))
        th = kz * st.layers[j - 1].h
        E = np.exp(-2j * th)
        tn[j], sc[j] = -1j * (1 - E) / (1 + E), 2 * np.exp(-1j * th) / (1 + E)
    Yd = [None] * (N + 1)
    Yd[1] = -1j * Y0[1] / tn[1]
    for k in range(2, N + 1):
        Yd[k] = Y0[k] * (Yd[k - 1] + 1j * Y0[k] * tn[k]) / (Y0[k] + 1j * Yd[k - 1] * tn[k])
    Yu = [None] * (N + 1)
    if st.top == 'open':
        Yu[N], kstart = y0(complex(st.top_er))[0], N
    else:
        Yu[N - 1], kstart = -1j * Y0[N] / tn[N], N - 1
    for k in range(kstart, 1, -1):
        Yu[k - 1] = Y0[k] * (Yu[k] + 1j * Y0[k] * tn[k]) / (Y0[k] + 1j * Yu[k] * tn[k])
    return Y0, tn, sc, Yd, Yu


def voltage(st, kr, w, o, s, mode):
    """multilayer.py:234-245: the voltage at interface o for a unit shunt current at interface s."""
    if st.is_pec(o) or st.is_pec(s):
        return np.zeros_like(np.asarray(kr, complex))
    Y0, tn, sc, Yd, Yu = network(st, kr, w, mode)
    v = 1.0 / (Yu[s] + Yd[s])
    for k in range(s + 1, o + 1):
        v = v * sc[k] / (1 + 1j * (Yu[k] / Y0[k]) * tn[k])
    for k in range(s, o, -1):
        v = v * sc[k] / (1 + 1j * (Yd[k - 1] / Y0[k]) * tn[k])
    return v


def spectral(st, kr, w, o, s):
    """multilayer.py:247-250: spectral G_A, G_q."""
    Vh, Ve = voltage(st, kr, w, o, s, 'h'), voltage(st, kr, w, o, s, 'e')
    return Vh / (1j * w), 1j * w * (Ve - Vh) / kr ** 2


def sommerfeld_contour(f, st, rho_max, K=None, nq=8):
    """via.py:36-53."""
    k0 = 2 * np.pi * f / C0
    kmax = k0 * np.sqrt(st.max_er())
    K = K or (max(1e5, 30.0 / st.hmin) + 40 * kmax)
    t1, alpha = 1.5 * kmax, min(0.5 * k0, 4.0 / rho_max)
    wid1, wid2 = min(0.3 * k0, 0.8 * alpha), 2 * np.pi / rho_max
    b1 = np.linspace(0, t1, int(np.ceil(t1 / wid1)) + 1)
    b2 = np.append(np.arange(t1, K, wid2), K)
    br = np.concatenate([b1, b2[1:]])
    xg, wg = np.polynomial.legendre.leggauss(nq)
    a, b = br[:-1, None], br[1:, None]
    t = (0.5 * (b - a) * xg[None, :] + 0.5 * (a + b)).ravel()
    wt = (0.5 * (b - a) * wg[None, :]).ravel()
    s = np.where(t < t1, alpha * np.sin(np.pi * t / t1), 0.0)
    ds = np.where(t < t1, alpha * np.pi / t1 * np.cos(np.pi * t / t1), 0.0)
    return t + 1j * s, wt * (1 + 1j * ds), K


def j0_sum(rho, kr, W):
    """via.py:90-101: sum_k J0(rho_i kr_k) W[s, k], the real part with glibc's j0, the lifted part complex."""
    rho, W = np.atleast_1d(np.asarray(rho, float)), np.atleast_2d(np.asarray(W, complex))
    real = np.abs(kr.imag) < 1e-300
    out = hankel_real(rho, np.ascontiguousarray(kr.real[real]), np.ascontiguousarray(W[:, real]))
    if (~real).any():
        out = out + (bessel_jn_complex(0, rho[:, None] * kr[None, ~real]) @ W[:, ~real].T).T
    return out


def hankel(spec, kr, dk, rho):
    """via.py:104-108: (1/2 pi) int spec J0(kr rho) kr dkr."""
    spec = np.asarray(spec)
    out = j0_sum(rho, kr, np.atleast_2d(spec) * (kr * dk)[None, :]) / (2 * np.pi)
    return out[0] if spec.ndim == 1 else out


class Table1D:
    """via.py:111-123: CubicSpline (not-a-knot) of vals on rho_coarse, resampled to nfine uniform points."""

    def __init__(self, rho_coarse, vals, rho_max, nfine=8192):
        self.rho = np.linspace(0, rho_max, nfine)
        self.v = CubicSpline(rho_coarse, vals)(self.rho)
        self._dr = self.rho[1]

    def __call__(self, r):
        u = np.minimum(np.asarray(r) / self._dr, len(self.rho) - 1.000001)
        i = u.astype(np.int64)
        t = (u - i).reshape(u.shape + (1,) * (self.v.ndim - 1))
        return self.v[i] * (1 - t) + self.v[i + 1] * t


class GreenTable:
    """multilayer.py:253-318."""

    def __init__(self, f, st, o, s, rho_max, nrho=260, nfine=8192, K=None, nq=8, cross_sing=False,
                 image_sing=None):
        w = 2 * np.pi * f
        self.o, self.s, self.f = o, s, f
        same, self.d = o == s, abs(st.z[o] - st.z[s])
        self.cA, self.cq = (MU0 / (4 * np.pi), 1.0 / (2 * np.pi * EPS0 * st.eps_sum(o))) if same else (0.0, 0.0)
        if cross_sing and not same:
            K1 = min(25.0 / st.hmin, 300.0 / self.d)
            ga, gq = spectral(st, np.array([K1 + 0j]), w, o, s)
            fac = K1 * np.exp(K1 * self.d) / (2 * np.pi)
            self.cA, self.cq = complex(ga[0] * fac), complex(gq[0] * fac)
        kr, dk, K = sommerfeld_contour(f, st, rho_max, K, nq)
        GA, Gq = spectral(st, kr, w, o, s)
        self.dimg, self.cAi, self.cqi = 0.0, 0.0, 0.0
        if same and image_sing:
            self.dimg = 2 * st.nearest_discontinuity(o)
            K1 = 18.0 / self.dimg
            ga, gq = spectral(st, np.array([K1 + 0j]), 2 * np.pi, o, s)
            fac = K1 * np.exp(K1 * self.dimg) / (2 * np.pi)
            self.cAi = complex((ga[0] - MU0 / (2 * K1)) * fac).real
            self.cqi = complex((gq[0] - 1.0 / (EPS0 * st.eps_sum(o) * K1)) * fac)
        for d, cA, cq in self.extracted():
            e = 2 * np.pi * np.exp(-kr * d) / kr
            GA, Gq = GA - cA * e, Gq - cq * e
        rho = rho_max * np.linspace(0, 1, nrho) ** 2
        self._tab = Table1D(rho, hankel(np.stack([GA, Gq]), kr, dk, rho).T, rho_max, nfine)
        self.rho, self.A_rest, self.Q_rest = self._tab.rho, self._tab.v[:, 0], self._tab.v[:, 1]
        self.npts, self.K, self.kr, self.dk = len(kr), K, kr, dk

    def extracted(self):
        if self.o != self.s:
            return [(self.d, self.cA, self.cq)] if self.cA != 0 else []
        return [(0.0, self.cA, self.cq)] + ([(self.dimg, self.cAi, self.cqi)] if self.dimg else [])

    def AQ(self, r):
        v = self._tab(r)
        return v[..., 0], v[..., 1]

    def total(self, rho):
        GA, GQ = self.AQ(rho)
        for d, cA, cq in self.extracted():
            R = np.hypot(rho, d)
            inv = np.divide(1.0, R, out=np.zeros(np.shape(R)), where=R > 0)
            GA, GQ = GA + cA * inv, GQ + cq * inv
        return GA, GQ


def green_tables(geo, f):
    """sim.py:736-745: {(a, b): GreenTable} for every pair of metal interfaces."""
    return {(a, b): GreenTable(f, geo.st, a, b, geo.rho_max, cross_sing=xs, image_sing=im)
            for a, b, xs, im in geo.table_pairs()}


def core_tables(geo, tables):
    """fast.py:556-568: the tb dictionary of the compiled core."""
    keys = sorted(tables)
    T = [tables[k] for k in keys]
    get = lambda attr, dt=float: np.array([dt(getattr(t, attr)) for t in T])
    return dict(A=np.stack([t.A_rest for t in T]).astype(complex), Q=np.stack([t.Q_rest for t in T]).astype(complex),
                dr=np.array([t.rho[1] for t in T]), d=get('d'), dimg=get('dimg'), cA=get('cA', complex),
                cq=get('cq', complex), cAi=get('cAi', complex), cqi=get('cqi', complex), tab=geo.tab_index(),
                kind=np.array([0 if a == b else (1 if t.cA != 0 else 2) for (a, b), t in zip(keys, T)], np.int32))
