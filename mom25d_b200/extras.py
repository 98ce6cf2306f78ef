"""
mom25d_b200.extras - the sparse additions to Z that the reference's FastOperator.extra_blocks makes
(fast.py:628-641):

  - series lumped elements across a strip (sim.py:221-226): Z(f) u u^T on the edges of the element's cut line,
    u = sign x length (sim.py:699-705, 726);
  - conductor loss (sim.py:228-270): the surface impedance Zs(f) times the RWG Gram matrix int f_m . f_n dS
    (base.py:153-157), row-scaled by Zs per edge where a surface finish covers some interfaces.

The Gram matrix and the element edges depend on the mesh only and are built once on the host, as the reference
caches its Gram matrix (sim._gram). Each frequency's values (a few scalars times those fixed patterns) go to the
device and are added into Z there by m25_coo_add, in FP64 for the double Z, rounded on store for complex64.
"""
import ctypes

import numpy as np

MU0 = 4e-7 * np.pi


def rlc(R=0.0, L=0.0, C=None, parallel=False):
    """The impedance function of a series (default) or parallel R-L-C element (sim.py:48-56)."""
    def Z(f):
        w = 2 * np.pi * f
        if not parallel:
            return R + 1j * w * L + (1 / (1j * w * C) if C else 0)
        return 1 / ((1 / R if R else 0) + (1 / (1j * w * L) if L else 0) + (1j * w * C if C else 0))
    return Z


def _zfun(Z):
    return Z if callable(Z) else (lambda f, Z=Z: complex(Z))


class SeriesLumped:
    """A series element across a strip (sim.py:221-226): the cut line of `width` at `center`, transverse to
    `direction`, on interface `layer`; Z an impedance (ohm) or a function of f (e.g. rlc(...))."""

    def __init__(self, layer, center, direction, width, Z, name=''):
        from .board import GapPort
        self.lp = GapPort(layer, center, direction, width, 0.0, name)   # the cut line's geometry
        self.layer, self.Z, self.name = int(layer), _zfun(Z), name


class Metal:
    """Conductor loss (sim.py:228-270): Zs = (g / sigma) coth(g t), g = (1 + j) / delta; rough (m RMS) scales its
    real part by Hammerstad and Jensen's 1 + 2/pi atan(1.4 (rough / delta)^2); finish [(sigma, t), ...] (outermost
    first) on the interfaces of `on` ({interface: share}) multiplies Zs there by 1 + share (F - 1), F the finished
    face's impedance over the bare one's."""

    def __init__(self, sigma=5.8e7, t=35e-6, rough=0.0, finish=(), on=None):
        self.sigma, self.t, self.rough = sigma, t, rough
        self.finish, self.on = [tuple(x) for x in finish], dict(on or {})

    def zs(self, f, k=None):
        g = (1 + 1j) * np.sqrt(2 * np.pi * f * MU0 * self.sigma / 2)
        z = g / self.sigma / np.tanh(g * self.t)
        if self.rough:
            delta = 1 / np.sqrt(np.pi * f * MU0 * self.sigma)
            z = z.real * (1 + 2 / np.pi * np.arctan(1.4 * (self.rough / delta) ** 2)) + 1j * z.imag
        share = self.on.get(k, 0.0) if self.finish else 0.0
        if share:
            z = z * (1 + share * (self.face_factor(f) - 1))
        return z

    def face_factor(self, f):
        """The finished face's impedance over the bare copper face's: each finish layer a line section
        Z_i = g_i / sigma_i loading the one beneath, from the copper outwards."""
        w = 2 * np.pi * f
        gam = lambda s: (1 + 1j) * np.sqrt(w * MU0 * s / 2)
        bare = gam(self.sigma) / self.sigma / np.tanh(gam(self.sigma) * self.t)
        z = bare
        for s, tl in reversed(self.finish):
            zc, th = gam(s) / s, np.tanh(gam(s) * tl)
            z = zc * (z + zc * th) / (zc + z * th)
        return z / bare

    def zs_edges(self, f, edge_layer):
        """Zs per RWG edge by its interface: one value unless a finish covers some interfaces."""
        if not (self.finish and self.on):
            return self.zs(f)
        out = np.full(len(edge_layer), self.zs(f), complex)
        for k in self.on:
            out[edge_layer == k] = self.zs(f, k)
        return out


def gram_matrix(rwg, P3, W3):
    """G[m, n] = int f_m . f_n dS (base.py:153-157) as (rows, cols, values) with unique (row, col): per triangle T
    and each pair of its RWG functions a, b (f = s l / (2 A) (r - v) on T), s_a s_b l_a l_b / (4 A) times the
    3-point rule's sum of (P_q - v_a) . (P_q - v_b) (exact: the integrand is quadratic)."""
    Ne, Nt = rwg.Ne, len(rwg.area)
    slot_rwg = np.full((Nt, 3), -1, np.int64)
    slot_sgn = np.zeros((Nt, 3))
    slot_v = np.zeros((Nt, 3, 2))
    fill = np.zeros(Nt, np.int64)
    for tri, sgn, v in ((rwg.tp, 1.0, rwg.vp), (rwg.tm, -1.0, rwg.vm)):
        for m in range(Ne):                                   # (a few slots a triangle: a plain loop is clear)
            t = tri[m]
            j = fill[t]
            slot_rwg[t, j], slot_sgn[t, j], slot_v[t, j] = m, sgn, v[m]
            fill[t] += 1
    A = rwg.area
    rows, cols, vals = [], [], []
    for a in range(3):
        for b in range(3):
            ok = (slot_rwg[:, a] >= 0) & (slot_rwg[:, b] >= 0)
            t = np.nonzero(ok)[0]
            ma, mb = slot_rwg[t, a], slot_rwg[t, b]
            da = P3[t] - slot_v[t, a][:, None, :]            # (nt, 3, 2)
            db = P3[t] - slot_v[t, b][:, None, :]
            q = (W3[None, :] * (da * db).sum(-1)).sum(1)
            rows.append(ma)
            cols.append(mb)
            vals.append(slot_sgn[t, a] * slot_sgn[t, b] * rwg.l[ma] * rwg.l[mb] / (4 * A[t]) * q)
    rows, cols, vals = np.concatenate(rows), np.concatenate(cols), np.concatenate(vals)
    key = rows * Ne + cols
    uk, inv = np.unique(key, return_inverse=True)
    v = np.zeros(len(uk))
    np.add.at(v, inv, vals)
    return (uk // Ne).astype(np.int64), (uk % Ne).astype(np.int64), v


class ExtraBlocks:
    """fast.py:628-641 for a Geometry: the fixed pattern (unique entries of Z that the lumped elements and the
    Gram matrix touch) and, per frequency, its values."""

    def __init__(self, geo, lumped=(), metal=None):
        self.geo, self.lumped, self.metal = geo, list(lumped), metal
        N, Ne = geo.N, geo.Ne
        parts_r, parts_c = [], []
        self.edges = []
        for el in self.lumped:                                # sim.py:726
            idx, sig = geo.gap_edges(el.lp)
            if not len(idx):
                raise ValueError(f"lumped element {el.name!r}: no mesh edges on its cut line")
            u = sig * geo.rwg.l[idx]
            self.edges.append((idx, u))
            parts_r.append(np.repeat(idx, len(idx)))
            parts_c.append(np.tile(idx, len(idx)))
        self.gram = None
        if metal is not None:
            from .board import BAR3, W3, quad_pts
            gr, gc, gv = gram_matrix(geo.rwg, quad_pts(geo.rwg, BAR3), W3)
            self.gram = (gr, gc, gv)
            parts_r.append(gr)
            parts_c.append(gc)
        if parts_r:
            r, c = np.concatenate(parts_r), np.concatenate(parts_c)
            key = np.unique(r * N + c)
        else:
            key = np.zeros(0, np.int64)
        self.ri, self.ci = (key // N).astype(np.int32), (key % N).astype(np.int32)
        self._key = key
        self._pos_lumped = [np.searchsorted(key, np.repeat(idx, len(idx)) * N + np.tile(idx, len(idx)))
                            for idx, _ in self.edges]
        self._pos_gram = None if self.gram is None else np.searchsorted(key, self.gram[0] * N + self.gram[1])
        self.edge_layer = geo.edge_layer
        self._dev = None

    @property
    def nnz(self):
        return len(self._key)

    def values(self, f):
        """The entries of S at f on the pattern (ri, ci): complex128[nnz]."""
        v = np.zeros(self.nnz, complex)
        for el, (idx, u), pos in zip(self.lumped, self.edges, self._pos_lumped):
            np.add.at(v, pos, el.Z(f) * np.outer(u, u).ravel())
        if self.gram is not None:
            zs = self.metal.zs_edges(f, self.edge_layer)
            gr, _, gv = self.gram
            np.add.at(v, self._pos_gram, (zs[gr] if np.ndim(zs) else zs) * gv)
        return v

    def dense(self, f):
        """S at f as a dense N x N array (tests)."""
        S = np.zeros((self.geo.N, self.geo.N), complex)
        S[self.ri, self.ci] = self.values(f)
        return S

    def add(self, Z, f, stream_ptr):
        """Z (a device complex128 or complex64 N x N tensor, row-major) += S at f, on the stream."""
        import torch
        from ._lib import P, check, lib
        if not self.nnz:
            return
        if self._dev is None:
            self._dev = (torch.from_numpy(self.ri).to('cuda'), torch.from_numpy(self.ci).to('cuda'))
        vv = torch.from_numpy(self.values(f)).to('cuda')
        single = int(Z.dtype == torch.complex64)
        check(lib().m25_coo_add(P(self._dev[0]), P(self._dev[1]), P(vv), ctypes.c_long(self.nnz), P(Z),
                                ctypes.c_long(Z.shape[1]), ctypes.c_int(Z.shape[0]), single, stream_ptr),
              'm25_coo_add')
        self._keep = vv                                       # until the stream has used it
