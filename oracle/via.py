"""
oracle.via - TEST INFRASTRUCTURE ONLY: NumPy restatement of the reference's via kernels and via blocks.

  TMNetwork       via.py:127-166   (TM voltages for every source interface)
  ViaKernels      via.py:179-235   (D tables per (interface, span), R via-via remainder, the homogeneous K0 term)
  via_blocks      sim.py:816-872   (B: Ne x Nv strip-via, C: Nv x Nv via-via, fan-distributed end charges)
  fan_columns     fast.py:489-504  (G_q moments to the fan triangles, near pairs corrected)
"""
import numpy as np
from scipy import sparse
from scipy.special import kv

from . import fan_q, radial_table_sum
from .green import MU0, C0, network, sommerfeld_contour, spectral, hankel, Table1D


class TMNetwork:
    def __init__(self, st, kr, w):
        self.st, self.kr, self.w, N = st, kr, w, st.N
        Y0, tn, sc, Yd, Yu = network(st, kr, w, 'e')
        self.k2 = [None] + [(w / C0) ** 2 * st.eps(j) for j in range(1, N + 1)]
        self.kz2 = [None] + [k2 - kr ** 2 for k2 in self.k2[1:]]
        self.V = {}
        for s in st.metal_interfaces:
            v = [None] * (N + 1)
            v[s] = 1.0 / (Yu[s] + Yd[s])
            for k in range(s + 1, N + 1):
                v[k] = np.zeros_like(kr) if st.is_pec(k) else v[k - 1] * sc[k] / (1 + 1j * (Yu[k] / Y0[k]) * tn[k])
            for k in range(s, 0, -1):
                v[k - 1] = np.zeros_like(kr) if st.is_pec(k - 1) else \
                    v[k] * sc[k] / (1 + 1j * (Yd[k - 1] / Y0[k]) * tn[k])
            self.V[s] = v

    def dV(self, i, s):
        return 0.0 if self.st.is_pec(s) else self.V[s][i] - self.V[s][i - 1]

    def S(self, k, layers):
        return sum((self.dV(j, k) / self.kz2[j] for j in layers), 0.0)

    def P(self, li, lj, with_homog=True):
        out = 0.0
        kr2 = self.kr ** 2
        for i in li:
            for j in lj:
                out = out + kr2 / (self.kz2[i] * self.kz2[j]) * (self.dV(i, j) - self.dV(i, j - 1))
                if with_homog and i == j:
                    out = out + 1j * self.w * MU0 * self.st.layers[j - 1].h / (kr2 - self.k2[j])
        return out


def chain_ends(k_bot, k_top):
    return [(k_bot, +1.0), (k_top, -1.0)]


def _layers(span):
    return range(span[0] + 1, span[1] + 1)


class ViaKernels:
    def __init__(self, f, st, spans, interfaces, rho_max, nrho=200):
        w = 2 * np.pi * f
        kr, dk, _ = sommerfeld_contour(f, st, rho_max)
        net = TMNetwork(st, kr, w)
        self.f, self.st, self.w, self.kr, self.dk, self.net = f, st, w, kr, dk, net
        self._gq = {}

        def gq(a, b):
            if st.is_pec(a) or st.is_pec(b):
                return 0.0
            key = (min(a, b), max(a, b))
            if key not in self._gq:
                self._gq[key] = spectral(st, kr, w, a, b)[1]
            return self._gq[key]
        self.gq, self.rho_max, self.D = gq, rho_max, {}
        rho = rho_max * np.linspace(0, 1, nrho) ** 2
        keys, specs = [], []
        for span in sorted(set(spans)):
            for k in interfaces:
                spec = net.S(k, _layers(span))
                for ke, div in chain_ends(*span):
                    spec = spec - div * gq(k, ke) / (1j * w)
                keys.append((k, span)); specs.append(spec * np.ones_like(kr))
        if keys:
            vals = hankel(np.array(specs), kr, dk, rho)
            for key, v in zip(keys, vals):
                self.D[key] = Table1D(rho, v, rho_max)

    def R(self, sm, sn, rho):
        spec = self.net.P(_layers(sm), _layers(sn), with_homog=False)
        for ka, da in chain_ends(*sm):
            for kb, db in chain_ends(*sn):
                spec = spec - da * db * self.gq(ka, kb) / (1j * self.w)
        return hankel(spec, self.kr, self.dk, rho)

    def R_table(self, sm, sn, nrho=200):
        rho = self.rho_max * np.linspace(0, 1, nrho) ** 2
        return Table1D(rho, self.R(sm, sn, rho), self.rho_max)

    def homog(self, sm, sn, rho):
        rho, out = np.atleast_1d(rho), np.zeros(np.size(rho), complex)
        for j in set(_layers(sm)) & set(_layers(sn)):
            kj = np.sqrt(self.net.k2[j] + 0j)
            if kj.imag > 0:
                kj = -kj
            out += 1j * self.w * MU0 * self.st.layers[j - 1].h / (2 * np.pi) * kv(0, 1j * kj * rho)
        return out


VIA_TABLE_PAIRS = 64


def divergence_T(geo, c):
    """r.D.T @ c: the RWG divergence (+l/A on T+, -l/A on T-) tested against per-triangle values c (Nt x k)."""
    r = geo.rwg
    return (2 * geo.h_alpha[:geo.Ne])[:, None] * c[r.tp] + (2 * geo.h_alpha[geo.Ne:])[:, None] * c[r.tm]


def fan_columns(geo, g, tb, nP, nQ, qcorr):
    """fast.py:489-504: the accurate G_q moments between every triangle and the fan triangles."""
    F = geo.F
    QF = fan_q(g, tb, np.asarray(F, np.int32))
    pos, sel = {q: j for j, q in enumerate(F)}, np.isin(nQ, F)
    np.add.at(QF, (nP[sel], np.array([pos[q] for q in nQ[sel]], int)), qcorr[sel])
    return QF


def via_blocks(geo, f, QF):
    """sim.py:816-872 (no frills, slots, lumped elements in vias or wall loss)."""
    w = 2 * np.pi * f
    B, C = np.zeros((geo.Ne, geo.Nv), complex), np.zeros((geo.Nv, geo.Nv), complex)
    vk = ViaKernels(f, geo.st, [(kb, kt) for _, kb, kt in geo.chains], geo.layers, geo.rho_max)
    if len(geo.F):
        dF = sparse.csc_matrix(geo.dF)
        T = np.asarray((dF.T @ QF.T).T)
        B += divergence_T(geo, T) / (1j * w)
        C += (dF.T @ T[geo.F]) / (1j * w)
    for span, ns in geo.by_span.items():
        c = np.zeros((geo.Nt, len(ns)), complex)
        for k in geo.layers:
            idx, D = geo.tri_idx[k], vk.D[(k, span)]
            c[idx] = radial_table_sum(geo.P6[idx, :, 0], geo.P6[idx, :, 1], geo.W6[idx], geo.ch_x[ns], geo.ch_y[ns],
                                      D.v, D._dr)
        B[:, ns] += divergence_T(geo, c)
    for (sm, sn), (m, n, dd) in geo.via_groups.items():
        vals = (vk.R_table(sm, sn)(dd) if len(dd) > VIA_TABLE_PAIRS else vk.R(sm, sn, dd)) + vk.homog(sm, sn, dd)
        C[m, n] += vals
        C[n[m != n], m[m != n]] += vals[m != n]
    return B, C, vk
