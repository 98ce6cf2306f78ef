"""
mom25d_b200.device - the per-frequency hot path on the GPU, orchestrated from the host: device-resident mesh
geometry, Green tables, via kernels and the impedance-matrix fill. Every arithmetic step runs in libmom25d_b200's
CUDA kernels; the host computes only parameters (the Sommerfeld contour's nodes, grids, index lists built once
per mesh) and reads back the handful of scalars the tables' singular coefficients need.

Layouts follow the reference (mom25d fast.py:377-406, 556-568): see geometry.py and include/mom25d_b200.h.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import P, check, lib, stream_ptr
from .board import MU0, C0, EPS0

c_int, c_long, c_double = ctypes.c_int, ctypes.c_long, ctypes.c_double

# multilayer.py:260 defaults; the mixed fill's complex64 tables keep the same grid (at 4096 points their linear
# interpolation differed from the double tables by ~1e-3 near rho = 0: too weak a preconditioner at low frequency)
TABLE_NRHO, TABLE_NFINE, TABLE_NFINE32 = 260, 8192, 8192
VIA_NRHO = 200                                                # via.py:179
VIA_TABLE_PAIRS = 64                                          # sim.py:784


def sommerfeld_contour(f, st, rho_max, K=None, nq=8):
    """Nodes and weights of the Sommerfeld integration path (via.py:36-53): lifted into the upper half plane by
    alpha sin up to 1.5 k_max, then real to K; Gauss-Legendre (nq points) on each piece."""
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


class _StackArgs:
    """The stack as the C ABI takes it (host arrays)."""

    def __init__(self, st):
        self.nl = st.N
        self.h = np.array([l.h for l in st.layers], float)
        self.eps = np.array([[st.eps(j).real, st.eps(j).imag] for j in range(1, st.N + 1)], float).ravel()
        self.top_open = 1 if st.top == 'open' else 0
        self.top_eps = np.array([st.top_er, 0.0])

    def args(self):
        return (c_int(self.nl), P(self.h), P(self.eps), c_int(self.top_open), P(self.top_eps))


class DeviceGeometry:
    """A Geometry (geometry.py) uploaded to the device, with the near pairs found there (once per mesh)."""

    def __init__(self, geo, stream=None):
        _lib.require_cuda()
        self.geo, self.stream = geo, stream
        d = _lib.dev
        g, q = geo.g, geo.q
        self.t = {k: d(g[k], np.int32 if k in ('ep', 'em', 'lt', 'te') else np.float64) for k in g}
        self.tq = {k: d(q[k], np.int32 if k == 'tris' else np.float64) for k in q}
        self.mesh = _lib.Mesh(geo.Ne, geo.Nt, *[P(self.t[k]) for k in ('ep', 'em', 'lt', 'te', 'ap', 'am', 'vp', 'vm',
                                                                          'cent', 'area', 'ta', 'tv')])
        self.quad = _lib.Quad(*[P(self.tq[k]) for k in ('nodes', 'tris', 'P3', 'W3', 'P6', 'W6')])
        self.size = d(geo.tri_size, np.float64)
        self.z = d(geo.tri_z, np.float64)
        self.stack = _StackArgs(geo.st)
        self._near_pairs()
        self.stat = torch.zeros(max(1, self.npairs) * 12, dtype=torch.float64, device='cuda')
        self.stat_ready = False
        self.rho_coarse = rho = geo.rho_max * np.linspace(0, 1, TABLE_NRHO) ** 2
        self.d_rho = d(rho)
        self.rho_via = geo.rho_max * np.linspace(0, 1, VIA_NRHO) ** 2
        self.d_rho_via = d(self.rho_via)
        self.tab = d(geo.tab_index(), np.int32)
        self._via_setup()

    def _near_pairs(self):
        geo = self.geo
        off = torch.zeros(geo.Nt + 1, dtype=torch.int64, device='cuda')
        total = ctypes.c_longlong(0)
        s = stream_ptr(self.stream)
        check(lib().m25_near_pairs(P(self.t['cent']), P(self.size), P(self.z), c_int(geo.Nt),
                                   c_double(geo.near_fac), P(off), ctypes.byref(total), ctypes.c_void_p(None),
                                   ctypes.c_void_p(None), s), 'm25_near_pairs')
        n = total.value
        self.nP = torch.empty(max(n, 1), dtype=torch.int32, device='cuda')
        self.nQ = torch.empty(max(n, 1), dtype=torch.int32, device='cuda')
        check(lib().m25_near_pairs(P(self.t['cent']), P(self.size), P(self.z), c_int(geo.Nt),
                                   c_double(geo.near_fac), P(off), ctypes.byref(total), P(self.nP), P(self.nQ), s),
              'm25_near_pairs')
        self.npairs = n
        self.off = off                                  # pairs of triangle p: off[p] .. off[p + 1] (sorted by p)

    def _via_setup(self):
        """Index lists of the via blocks, built once (sim.py:786-814): the fans' divergence dF as CSR by chain,
        the near pairs landing on a fan column, the via pairs by span pair."""
        geo = self.geo
        self.Nv = geo.Nv
        if not geo.Nv:
            return
        d = _lib.dev
        dF = geo.dF
        ptr, fj, fw = [0], [], []
        for n in range(geo.Nv):
            nz = np.flatnonzero(dF[:, n])
            fj += nz.tolist(); fw += dF[nz, n].tolist(); ptr.append(len(fj))
        self.v_ptr, self.v_fj, self.v_fw = d(np.array(ptr), np.int32), d(np.array(fj), np.int32), d(np.array(fw))
        self.v_F = d(geo.F, np.int32)
        self.nf = len(geo.F)
        nP, nQ = self.nP[:self.npairs].cpu().numpy(), self.nQ[:self.npairs].cpu().numpy()
        pos = -np.ones(geo.Nt, np.int64)
        pos[geo.F] = np.arange(len(geo.F))
        sel = np.flatnonzero(pos[nQ] >= 0)
        self.q_pair, self.q_row, self.q_col = d(sel, np.int32), d(nP[sel], np.int32), d(pos[nQ[sel]], np.int32)
        self.nq_sel = len(sel)
        # D tables: (interface, span) for every metal interface and span; a table index per (layer index, span)
        self.spans = geo.spans
        self.d_keys = [(k, sp) for sp in self.spans for k in geo.layers]       # via.py:205-211 order
        dtab = np.zeros((len(geo.layers), len(self.spans)), np.int32)
        for i, (k, sp) in enumerate(self.d_keys):
            dtab[geo.lidx[k], self.spans.index(sp)] = i
        self.v_dtab = d(dtab)
        span_of = np.array([self.spans.index((kb, kt)) for _, kb, kt in geo.chains], np.int32)
        self.v_span_of = d(span_of)
        self.v_x, self.v_y = d(geo.ch_x), d(geo.ch_y)
        self.groups = []
        for (sm, sn), (m, n, dd) in geo.via_groups.items():
            mask = 0
            for j in set(range(sm[0] + 1, sm[1] + 1)) & set(range(sn[0] + 1, sn[1] + 1)):
                mask |= 1 << j
            self.groups.append(dict(sm=sm, sn=sn, m=d(m, np.int32), n=d(n, np.int32), dd=d(dd), np=len(dd),
                                    mask=mask, table=len(dd) > VIA_TABLE_PAIRS))


class DeviceTables:
    """The Green tables of one frequency on the device (multilayer.py:253-318 for every interface pair, packed as
    fast.py:556-568): complex128 tables of TABLE_NFINE samples for the double-precision path, and complex64 ones of
    TABLE_NFINE32 for the mixed-precision fill."""

    def __init__(self, dg, f, single=False, stream=None):
        geo, st = dg.geo, dg.geo.st
        self.f, self.w = f, 2 * np.pi * f
        w = self.w
        s = stream_ptr(stream)
        pairs = geo.table_pairs()
        npair = len(pairs)
        # singular coefficients: same interface analytic; the large-kr limits from the network on the GPU
        cA = np.zeros(npair, complex); cq = np.zeros(npair, complex)
        cAi = np.zeros(npair, complex); cqi = np.zeros(npair, complex)
        dd = np.zeros(npair); dimg = np.zeros(npair)
        ext = []
        for i, (a, b, xs, im) in enumerate(pairs):
            same = a == b
            dd[i] = abs(st.z[a] - st.z[b])
            if same:
                cA[i], cq[i] = MU0 / (4 * np.pi), 1.0 / (2 * np.pi * EPS0 * st.eps_sum(a))
            if xs and not same:
                K1 = min(25.0 / st.hmin, 300.0 / dd[i])
                ext.append((i, 'x', K1, w))
            if same and im:
                dimg[i] = 2 * st.nearest_discontinuity(a)
                ext.append((i, 'i', 18.0 / dimg[i], 2 * np.pi))
        if ext:
            kr = _lib.dev(np.array([e[2] for e in ext], complex))
            ww = _lib.dev(np.array([e[3] for e in ext], float))
            ga = torch.empty(len(ext), dtype=torch.complex128, device='cuda')
            gq = torch.empty_like(ga)
            for j, (i, kind, K1, wj) in enumerate(ext):
                a, b = pairs[i][0], pairs[i][1]
                check(lib().m25_spectral_points(P(kr[j:]), P(ww[j:]), c_int(1), *dg.stack.args(), c_int(a), c_int(b),
                                                P(ga[j:]), P(gq[j:]), s), 'm25_spectral_points')
            ga, gq = ga.cpu().numpy(), gq.cpu().numpy()
            for j, (i, kind, K1, wj) in enumerate(ext):
                a = pairs[i][0]
                if kind == 'x':
                    fac = K1 * np.exp(K1 * dd[i]) / (2 * np.pi)
                    cA[i], cq[i] = complex(ga[j] * fac), complex(gq[j] * fac)
                else:
                    fac = K1 * np.exp(K1 * dimg[i]) / (2 * np.pi)
                    cAi[i] = complex((ga[j] - MU0 / (2 * K1)) * fac).real
                    cqi[i] = complex((gq[j] - 1.0 / (EPS0 * st.eps_sum(a) * K1)) * fac)
        kind = np.array([0 if a == b else (1 if cA[i] != 0 else 2) for i, (a, b, _, _) in enumerate(pairs)], np.int32)
        nxt = np.zeros(npair, np.int32)
        ed = np.zeros((npair, 2)); ecA = np.zeros((npair, 2), complex); ecq = np.zeros((npair, 2), complex)
        for i, (a, b, _, _) in enumerate(pairs):                # multilayer.py:294-299 extracted()
            lst = ([(dd[i], cA[i], cq[i])] if cA[i] != 0 else []) if a != b else \
                [(0.0, cA[i], cq[i])] + ([(dimg[i], cAi[i], cqi[i])] if dimg[i] else [])
            nxt[i] = len(lst)
            for j, (x, y, z) in enumerate(lst):
                ed[i, j], ecA[i, j], ecq[i, j] = x, y, z
        # the contour and the spectra with the extracted parts removed
        krh, dkh, K = sommerfeld_contour(f, st, geo.rho_max)
        self.npts = npts = len(krh)
        d_kr, d_dk = _lib.dev(krh), _lib.dev(dkh)
        W = torch.empty((2 * npair, npts), dtype=torch.complex128, device='cuda')   # GA rows, then GQ rows
        scratch = torch.empty(int(lib().m25_pair_record_bytes()), dtype=torch.uint8, device='cuda')
        h_o = np.array([p[0] for p in pairs], np.int32)      # (host arrays kept alive across the call)
        h_s = np.array([p[1] for p in pairs], np.int32)
        check(lib().m25_spectral_extracted(P(d_kr), c_int(npts), c_double(w), *dg.stack.args(), c_int(npair),
                                           P(h_o), P(h_s), P(nxt), P(ed.ravel()),
                                           P(np.ascontiguousarray(ecA).view(float).ravel()),
                                           P(np.ascontiguousarray(ecq).view(float).ravel()), P(W), P(W[npair:]),
                                           P(scratch), s), 'm25_spectral_extracted')
        H = torch.empty((2 * npair, TABLE_NRHO), dtype=torch.complex128, device='cuda')
        for r0 in range(0, 2 * npair, 16):
            r1 = min(2 * npair, r0 + 16)
            check(lib().m25_hankel(P(d_kr), P(d_dk), c_int(npts), P(W[r0:]), c_int(r1 - r0), P(dg.d_rho),
                                   c_int(TABLE_NRHO), P(H[r0:]), s), 'm25_hankel')
        self.H = H
        rho_max = geo.rho_max
        nf = TABLE_NFINE
        dx = np.linspace(0, rho_max, nf)[1]
        self.AQ = torch.empty((2 * npair, nf), dtype=torch.complex128, device='cuda')
        check(lib().m25_spline_uniform(P(dg.d_rho), P(H), c_int(2 * npair), c_int(TABLE_NRHO), c_double(dx), c_int(nf),
                                       P(self.AQ), c_int(0), c_long(nf), c_long(0), c_int(1), s), 'm25_spline_uniform')
        self.scal = _lib.dev(np.concatenate([cA, cq, cAi, cqi]))
        self.dr = _lib.dev(np.full(npair, dx))
        self.d = _lib.dev(dd)
        self.dimg = _lib.dev(dimg)
        self.kind = _lib.dev(kind)
        self.host = dict(cA=cA, cq=cq, cAi=cAi, cqi=cqi, d=dd, dimg=dimg, kind=kind, dr=np.full(npair, dx))
        self.tables = _lib.Tables(npair, nf, len(geo.layers), P(self.AQ), P(self.AQ[npair:]), P(self.scal),
                                  P(self.scal[npair:]), P(self.scal[2 * npair:]), P(self.scal[3 * npair:]),
                                  P(self.dr), P(self.d), P(self.dimg), P(dg.tab), P(self.kind))
        self.kr, self.dk, self.d_kr, self.d_dk = krh, dkh, d_kr, d_dk
        self.tables32 = None
        if single:
            nf32 = TABLE_NFINE32
            dx32 = np.linspace(0, rho_max, nf32)[1]
            self.AQ32 = torch.empty((2 * npair, nf32), dtype=torch.complex64, device='cuda')
            check(lib().m25_spline_uniform(P(dg.d_rho), P(H), c_int(2 * npair), c_int(TABLE_NRHO), c_double(dx32),
                                           c_int(nf32), P(self.AQ32), c_int(1), c_long(nf32), c_long(0), c_int(1), s),
                  'm25_spline_uniform')
            self.scal32 = self.scal.to(torch.complex64)
            self.f32 = _lib.dev(np.concatenate([np.full(npair, dx32), dd, dimg]), np.float32)
            self.tables32 = _lib.TablesF(npair, nf32, len(geo.layers), P(self.AQ32), P(self.AQ32[npair:]),
                                         P(self.scal32), P(self.scal32[npair:]), P(self.scal32[2 * npair:]),
                                         P(self.scal32[3 * npair:]), P(self.f32), P(self.f32[npair:]),
                                         P(self.f32[2 * npair:]), P(dg.tab), P(self.kind))

    def host_dict(self, geo):
        """The tables as the reference core's tb dictionary (host copies), for checks."""
        n = len(self.host['kind'])
        AQ = self.AQ.cpu().numpy()
        return dict(A=AQ[:n], Q=AQ[n:], tab=geo.tab_index(), **self.host)


class DeviceVias:
    """The via rows and columns of one frequency (sim.py:816-872) on the device, written into Z."""

    def __init__(self, dg, tabs, stream=None):
        self.dg, self.tabs, geo = dg, tabs, dg.geo
        self.stream = stream

    def assemble(self, Z, ld, qcorr, Z64=None, B=None, C=None):
        """Writes the border into Z (complex128) and / or Z64 (complex64), and B, C when given."""
        dg, geo, tb = self.dg, self.dg.geo, self.tabs
        if not geo.Nv:
            return
        s = stream_ptr(self.stream)
        w = tb.w
        Nt, Nv, nf = geo.Nt, geo.Nv, dg.nf
        # fan columns (fast.py:489-504) and the fan-charge potential T (sim.py:839-843)
        QF = torch.empty((Nt, nf), dtype=torch.complex128, device='cuda')
        check(lib().m25_fan_q(P(dg.v_F), c_int(nf), P(QF), ctypes.byref(dg.mesh), ctypes.byref(tb.tables), s),
              'm25_fan_q')
        check(lib().m25_via_qcorr(P(QF), c_int(nf), P(dg.q_pair), P(dg.q_row), P(dg.q_col), c_int(dg.nq_sel),
                                  P(qcorr), s), 'm25_via_qcorr')
        T = torch.empty((Nt, Nv), dtype=torch.complex128, device='cuda')
        check(lib().m25_via_fan_T(P(QF), c_int(Nt), c_int(nf), P(dg.v_ptr), P(dg.v_fj), P(dg.v_fw), c_int(Nv), P(T), s),
              'm25_via_fan_T')
        # via spectra: D(k, span) then R for every span pair of the groups (via.py:195-222)
        dk = np.array([k for k, _ in dg.d_keys], np.int32)
        dspan = np.array([sp for _, sp in dg.d_keys], np.int32).ravel()
        rm = np.array([g['sm'] for g in dg.groups], np.int32).ravel()
        rn = np.array([g['sn'] for g in dg.groups], np.int32).ravel()
        nd, nr = len(dg.d_keys), len(dg.groups)
        npts = tb.npts
        spec = torch.empty((nd + nr, npts), dtype=torch.complex128, device='cuda')
        check(lib().m25_via_spectra(P(tb.d_kr), c_int(npts), c_double(w), *dg.stack.args(), c_int(nd), P(dk), P(dspan),
                                    c_int(nr), P(rm), P(rn), P(spec), s), 'm25_via_spectra')
        # D tables: Hankel on the via grid, spline to 8192 points (via.py:210-213, Table1D)
        Hd = torch.empty((nd, VIA_NRHO), dtype=torch.complex128, device='cuda')
        for r0 in range(0, nd, 16):
            r1 = min(nd, r0 + 16)
            check(lib().m25_hankel(P(tb.d_kr), P(tb.d_dk), c_int(npts), P(spec[r0:]), c_int(r1 - r0),
                                   P(dg.d_rho_via), c_int(VIA_NRHO), P(Hd[r0:]), s), 'm25_hankel')
        nfv = TABLE_NFINE
        dxv = np.linspace(0, geo.rho_max, nfv)[1]
        D = torch.empty((nd, nfv), dtype=torch.complex128, device='cuda')
        check(lib().m25_spline_uniform(P(dg.d_rho_via), P(Hd), c_int(nd), c_int(VIA_NRHO), c_double(dxv), c_int(nfv),
                                       P(D), c_int(0), c_long(nfv), c_long(0), c_int(1), s), 'm25_spline_uniform')
        c = torch.empty((Nt, Nv), dtype=torch.complex128, device='cuda')
        check(lib().m25_via_radial(P(dg.tq['P6']), P(dg.tq['W6']), P(dg.t['lt']), c_int(Nt), P(dg.v_x), P(dg.v_y),
                                   P(dg.v_span_of), c_int(Nv), P(D), P(dg.v_dtab), c_int(len(dg.spans)), c_long(nfv),
                                   c_double(dxv), P(c), s), 'm25_via_radial')
        # via-via remainder R (exact at the pairs' distances, or its table for many pairs) + K0 part (sim.py:862-866)
        R = torch.zeros((Nv, Nv), dtype=torch.complex128, device='cuda')
        for j, gr in enumerate(dg.groups):
            hom = torch.empty(gr['np'], dtype=torch.complex128, device='cuda')
            check(lib().m25_via_homog(P(gr['dd']), c_int(gr['np']), c_double(w), *dg.stack.args(), ctypes.c_uint(gr['mask']),
                                      P(hom), s), 'm25_via_homog')
            if gr['table']:
                Hr = torch.empty((1, VIA_NRHO), dtype=torch.complex128, device='cuda')
                check(lib().m25_hankel(P(tb.d_kr), P(tb.d_dk), c_int(npts), P(spec[nd + j:]), c_int(1),
                                       P(dg.d_rho_via), c_int(VIA_NRHO), P(Hr), s), 'm25_hankel')
                Rt = torch.empty((1, nfv), dtype=torch.complex128, device='cuda')
                check(lib().m25_spline_uniform(P(dg.d_rho_via), P(Hr), c_int(1), c_int(VIA_NRHO), c_double(dxv),
                                               c_int(nfv), P(Rt), c_int(0), c_long(nfv), c_long(0), c_int(1), s),
                      'm25_spline_uniform')
                check(lib().m25_via_pairs(P(gr['m']), P(gr['n']), P(gr['dd']), c_int(gr['np']), P(None), P(hom), P(Rt),
                                          c_long(nfv), c_double(dxv), c_int(Nv), P(R), s), 'm25_via_pairs')
            else:
                vals = torch.empty((1, gr['np']), dtype=torch.complex128, device='cuda')
                check(lib().m25_hankel(P(tb.d_kr), P(tb.d_dk), c_int(npts), P(spec[nd + j:]), c_int(1), P(gr['dd']),
                                       c_int(gr['np']), P(vals), s), 'm25_hankel')
                check(lib().m25_via_pairs(P(gr['m']), P(gr['n']), P(gr['dd']), c_int(gr['np']), P(vals), P(hom),
                                          P(None), c_long(0), c_double(0), c_int(Nv), P(R), s), 'm25_via_pairs')
        check(lib().m25_via_assemble(P(T), P(c), P(dg.v_F), P(dg.v_ptr), P(dg.v_fj), P(dg.v_fw), c_int(Nv), P(R),
                                     ctypes.byref(dg.mesh), c_double(w), P(Z), P(Z64), c_long(ld), P(B), P(C), s),
              'm25_via_assemble')
        self.keep = (QF, T, spec, Hd, D, c, R)
