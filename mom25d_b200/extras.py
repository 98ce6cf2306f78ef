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
    """Z(f) of an R-L-C element, the reference's rlc (sim.py:51-58) by its definition: in series the branch
    impedances R, j w L and 1 / (j w C) add (no C: no capacitor in the string); in parallel their admittances
    add, a zero R or L or a missing C being an absent branch."""
    if parallel:
        def Z(f):
            jw = 2j * np.pi * f
            y = 0.0
            if R:
                y += 1.0 / R
            if L:
                y += 1.0 / (jw * L)
            if C:
                y += jw * C
            return 1.0 / y
    else:
        def Z(f):
            jw = 2j * np.pi * f
            z = R + jw * L
            return z + 1.0 / (jw * C) if C else z
    return Z


def as_impedance(Z):
    """An impedance given as ohms or as a function of f, as a function of f."""
    if callable(Z):
        return Z
    z = complex(Z)
    return lambda f: z


class SeriesLumped:
    """A series element across a strip (sim.py:221-226): the cut line of `width` at `center`, transverse to
    `direction`, on interface `layer`; Z an impedance (ohm) or a function of f (e.g. rlc(...)). The reference's
    own SeriesLumped objects work here as well (the same .lp cut line and .Z)."""

    def __init__(self, layer, center, direction, width, Z, name=''):
        from .board import GapPort
        self.lp = GapPort(layer, center, direction, width, 0.0, name)   # the cut line's geometry
        self.layer, self.Z, self.name = int(layer), as_impedance(Z), name


def _skin_wavenumber(w, sigma):
    """(1 + j) / delta, delta = sqrt(2 / (w mu0 sigma)) the skin depth of a good conductor at angular frequency w."""
    return (1.0 + 1.0j) * np.sqrt(0.5 * w * MU0 * sigma)


def _slab_impedance(w, sigma, t):
    """The surface impedance of a conductor slab of thickness t seen from one face: Zc coth(gamma t) with the
    wave impedance Zc = gamma / sigma of the conductor (tends to 1 / (sigma t) at DC)."""
    gm = _skin_wavenumber(w, sigma)
    return (gm / sigma) / np.tanh(gm * t)


def _through_layer(z_load, w, sigma, t):
    """The impedance at the outer face of a finish layer (sigma, t) backed by z_load: the layer as a line section
    of wave impedance Zc = gamma / sigma and electrical length gamma t terminated in z_load."""
    gm = _skin_wavenumber(w, sigma)
    zc, th = gm / sigma, np.tanh(gm * t)
    return zc * (z_load + zc * th) / (zc + z_load * th)


class Metal:
    """Conductor loss of the strips (the reference's Metal, sim.py:228-270): the surface impedance Zs of a copper
    slab (sigma, t), its resistance scaled by Hammerstad and Jensen's roughness factor for an RMS roughness
    `rough`, and where a surface finish ([(sigma, t), ...], outermost first) covers the interfaces of `on`
    ({interface: share}), Zs there scaled by 1 + share (F - 1), F the finished face over the bare face. The
    reference's own Metal objects work here as well (the same zs_edges)."""

    def __init__(self, sigma=5.8e7, t=35e-6, rough=0.0, finish=(), on=None):
        self.sigma, self.t, self.rough = sigma, t, rough
        self.finish, self.on = [tuple(x) for x in finish], dict(on or {})

    def roughness_factor(self, f):
        """1 + (2 / pi) atan(1.4 (rough / delta)^2), delta the copper's skin depth at f (1 when smooth)."""
        if not self.rough:
            return 1.0
        delta = np.sqrt(1.0 / (np.pi * f * MU0 * self.sigma))
        return 1.0 + (2.0 / np.pi) * np.arctan(1.4 * (self.rough / delta) ** 2)

    def face_factor(self, f):
        """The finished face's impedance over the bare copper face's at f: the finish layers stacked on the
        copper slab from the innermost outwards."""
        w = 2 * np.pi * f
        bare = _slab_impedance(w, self.sigma, self.t)
        z = bare
        for sigma, t in self.finish[::-1]:
            z = _through_layer(z, w, sigma, t)
        return z / bare

    def zs(self, f, k=None):
        """Zs at f, on interface k (its finish, if any)."""
        z = _slab_impedance(2 * np.pi * f, self.sigma, self.t)
        kr = self.roughness_factor(f)
        if kr != 1.0:
            z = complex(z.real * kr, z.imag)
        share = self.on.get(k, 0.0) if self.finish else 0.0
        if share:
            z = z * (1.0 + share * (self.face_factor(f) - 1.0))
        return z

    def zs_edges(self, f, edge_layer):
        """Zs for every RWG edge by its interface: a scalar when no finish is set on some interfaces."""
        if not (self.finish and self.on):
            return self.zs(f)
        edge_layer = np.asarray(edge_layer)
        ks = np.unique(edge_layer)
        per = np.array([self.zs(f, int(k)) if int(k) in self.on else self.zs(f) for k in ks], complex)
        return per[np.searchsorted(ks, edge_layer)]


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

    def _device_values(self, f, stream):
        """The pattern (ri, ci) and S's values at f as device tensors, uploaded on `stream` (a torch stream, or
        None for the current one) so that the caching allocator hands their memory on only after that stream has
        used them; the values are kept for the frequency until another is asked for."""
        import torch
        st = stream if stream is not None else torch.cuda.current_stream()
        with torch.cuda.stream(st):
            if self._dev is None:
                self._dev = (torch.from_numpy(self.ri).to('cuda'), torch.from_numpy(self.ci).to('cuda'))
            if getattr(self, '_vals_f', None) != f:
                self._vals = torch.from_numpy(self.values(f)).to('cuda')
                self._vals_f = f
        return self._dev[0], self._dev[1], self._vals

    def add(self, Z, f, stream=None):
        """Z (a device complex128 or complex64 N x N tensor, row-major) += S at f, on the stream (a torch stream,
        or None for the current one)."""
        import torch
        from ._lib import P, check, lib, stream_ptr
        if not self.nnz:
            return
        ri, ci, vv = self._device_values(f, stream)
        single = int(Z.dtype == torch.complex64)
        check(lib().m25_coo_add(P(ri), P(ci), P(vv), ctypes.c_long(self.nnz), P(Z), ctypes.c_long(Z.shape[1]),
                                ctypes.c_int(Z.shape[0]), single, stream_ptr(stream)), 'm25_coo_add')

    def apply(self, X, Y, f, stream=None):
        """Y += S X at f (X, Y device complex128 N x k, contiguous): the extra blocks in the matrix-free
        refinement operator, as the reference's matvec_exact adds Sx X (fast.py:571-586)."""
        from ._lib import P, check, lib, stream_ptr
        if not self.nnz:
            return
        ri, ci, vv = self._device_values(f, stream)
        check(lib().m25_coo_spmm(P(ri), P(ci), P(vv), ctypes.c_long(self.nnz), P(X), ctypes.c_int(X.shape[1]), P(Y),
                                 stream_ptr(stream)), 'm25_coo_spmm')
