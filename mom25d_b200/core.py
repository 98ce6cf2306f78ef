"""
mom25d_b200.core - a drop-in for the reference's compiled kernel module (mom25d `_core`, chosen by
fast.use_core / fast.set_core, fast.py:27-51): the same function names, arguments, return values and in-place
semantics (pybind11 signatures, mom25d_core.cpp:1658-1702), each running on the GPU through libmom25d_b200.

    import mom25d.fast as fast, mom25d_b200.core as core
    fast.set_core(core)            # every fill / near / via / Hankel call of the reference now runs on the B200

Host NumPy arrays in and out, as the reference's module takes them: each call uploads what it reads, runs the
kernels on the current CUDA stream and copies its results back before it returns (the reference's calls are
synchronous too). Arrays the reference writes in place (Z, q['stat']) are written in place. Bad shapes raise
ValueError, as pybind11 turns the core's std::invalid_argument into; a CUDA or kernel error raises M25Error (a
RuntimeError). There is no CPU path: without a CUDA device every call raises.

The device-resident path (fill into a device Z, LU and solves without a host round trip) is
mom25d_b200.operator.DirectSolver; this module is the per-call boundary.
"""
import ctypes
import os

import numpy as np
import torch

from . import _lib
from ._lib import P, check, lib, stream_ptr

c_int, c_long, c_double = ctypes.c_int, ctypes.c_long, ctypes.c_double

_MESH_INT = ('ep', 'em', 'lt', 'te')
_MESH_F64 = ('ap', 'am', 'vp', 'vm', 'cent', 'area', 'ta', 'tv')


class _Dev:
    """Device copies of one call's arguments (kept alive until the call returns)."""

    def __init__(self):
        _lib.require_cuda()
        self.keep = []

    def put(self, a, dtype):
        t = _lib.dev(a, dtype)
        self.keep.append(t)
        return t

    def mesh(self, g):
        for k in _MESH_INT + _MESH_F64:
            if k not in g:
                raise ValueError(f"geometry dict: missing {k!r}")
        t = {k: self.put(g[k], np.int32 if k in _MESH_INT else np.float64) for k in _MESH_INT + _MESH_F64}
        Ne, Nt = len(g['ep']), len(g['lt'])
        if len(g['em']) != Ne or np.size(g['te']) != 3 * Nt or np.size(g['tv']) != 6 * Nt:
            raise ValueError("geometry dict: inconsistent edge / triangle array sizes")
        return _lib.Mesh(Ne, Nt, *[P(t[k]) for k in ('ep', 'em', 'lt', 'te', 'ap', 'am', 'vp', 'vm', 'cent', 'area',
                                                      'ta', 'tv')])

    def tables(self, tb):
        for k in ('A', 'Q', 'cA', 'cq', 'cAi', 'cqi', 'dr', 'd', 'dimg', 'tab', 'kind'):
            if k not in tb:
                raise ValueError(f"tables dict: missing {k!r}")
        A = np.asarray(tb['A'])
        if A.ndim != 2 or np.shape(tb['Q']) != A.shape:
            raise ValueError("tables dict: A and Q must be (ntab, nfine)")
        tab = np.asarray(tb['tab'])
        d = {k: self.put(tb[k], np.complex128) for k in ('A', 'Q', 'cA', 'cq', 'cAi', 'cqi')}
        d.update({k: self.put(tb[k], np.float64) for k in ('dr', 'd', 'dimg')})
        d.update({k: self.put(tb[k], np.int32) for k in ('tab', 'kind')})
        return _lib.Tables(A.shape[0], A.shape[1], tab.shape[0],
                           *[P(d[k]) for k in ('A', 'Q', 'cA', 'cq', 'cAi', 'cqi', 'dr', 'd', 'dimg', 'tab', 'kind')])

    def quad(self, q):
        for k in ('nodes', 'tris', 'P3', 'W3', 'P6', 'W6'):
            if k not in q:
                raise ValueError(f"quad dict: missing {k!r}")
        t = {k: self.put(q[k], np.int32 if k == 'tris' else np.float64) for k in ('nodes', 'tris', 'P3', 'W3', 'P6',
                                                                                   'W6')}
        return _lib.Quad(*[P(t[k]) for k in ('nodes', 'tris', 'P3', 'W3', 'P6', 'W6')])


def _done(what):
    _lib.sync_check(what=what)


def _z_matrix(Z, Ne):
    if not isinstance(Z, np.ndarray) or Z.ndim != 2 or not Z.flags.c_contiguous:
        raise ValueError("Z must be a C-contiguous 2-D array")
    if Z.dtype not in (np.complex128, np.complex64):
        raise ValueError("Z must be complex128 or complex64")
    if Z.shape[0] < Ne or Z.shape[1] < Ne:
        raise ValueError(f"Z ({Z.shape}) is smaller than the {Ne} edges")


# ---- the far field (mom25d_core.cpp:132-314) ----------------------------------------------------------------------
def fill_far(Z, g, tb, w):
    """Far-field (centroid rule) entries of every edge pair into Z[:Ne, :Ne], both triangles and the diagonal
    written (mom25d_core.cpp:132-173). Z complex128 (or complex64: the FP64 values rounded on store, as the
    reference's fill_far_c64)."""
    D = _Dev()
    Ne = len(g['ep'])
    _z_matrix(Z, Ne)
    m, t = D.mesh(g), D.tables(tb)
    Zd = torch.empty((Ne, Ne), dtype=torch.complex128, device='cuda')
    check(lib().m25_fill_far(P(Zd), c_long(Ne), 0, ctypes.byref(m), ctypes.byref(t), None, c_double(w),
                             stream_ptr()), 'fill_far')
    if Z.dtype == np.complex64:
        Zf = torch.empty((Ne, Ne), dtype=torch.complex64, device='cuda')
        check(lib().m25_convert(P(Zd), 0, P(Zf), c_long(Ne * Ne), stream_ptr()), 'fill_far_c64')
        Zd = Zf
    _done('fill_far')
    Z[:Ne, :Ne] = Zd.cpu().numpy()


def fill_far_c64(Z, g, tb, w):
    if Z.dtype != np.complex64:
        raise ValueError("fill_far_c64: Z must be complex64")
    fill_far(Z, g, tb, w)


def far_block(rows, cols, g, tb, w):
    """The far field of row edges x column edges: complex128 (nr, nc) (mom25d_core.cpp:176-211)."""
    D = _Dev()
    rows, cols = np.ascontiguousarray(rows, np.int32), np.ascontiguousarray(cols, np.int32)
    Ne = len(g['ep'])
    if rows.size and (rows.min() < 0 or rows.max() >= Ne) or cols.size and (cols.min() < 0 or cols.max() >= Ne):
        raise ValueError("far_block: edge index out of range")
    m, t = D.mesh(g), D.tables(tb)
    out = torch.zeros((len(rows), len(cols)), dtype=torch.complex128, device='cuda')
    check(lib().m25_far_block(P(D.put(rows, np.int32)), c_int(len(rows)), P(D.put(cols, np.int32)), c_int(len(cols)),
                              P(out), ctypes.byref(m), ctypes.byref(t), c_double(w), stream_ptr()), 'far_block')
    _done('far_block')
    return out.cpu().numpy()


def matvec_far_multi(X, g, tb, w):
    """Y = Z_far X for the columns of X (Ne, k) without Z (mom25d_core.cpp:257-314)."""
    D = _Dev()
    X = np.ascontiguousarray(X, np.complex128)
    Ne, Nt = len(g['ep']), len(g['lt'])
    if X.ndim != 2 or X.shape[0] != Ne:
        raise ValueError(f"matvec_far_multi: X must be ({Ne}, k)")
    k = X.shape[1]
    m, t = D.mesh(g), D.tables(tb)
    Xd = D.put(X, np.complex128)
    Y = torch.empty_like(Xd)
    work = torch.empty(6 * Nt * max(k, 1), dtype=torch.complex128, device='cuda')
    if k:
        check(lib().m25_matvec_far_multi(P(Xd), c_int(k), P(Y), P(work), ctypes.byref(m), ctypes.byref(t),
                                         c_double(w), stream_ptr()), 'matvec_far_multi')
    _done('matvec_far_multi')
    return Y.cpu().numpy()


def matvec_far(x, g, tb, w):
    """One column of matvec_far_multi (mom25d_core.cpp:214)."""
    return matvec_far_multi(np.asarray(x, np.complex128).reshape(-1, 1), g, tb, w)[:, 0]


# ---- the near field (mom25d_core.cpp:417-579) ---------------------------------------------------------------------
def _near(mode, Z, g, tb, q, Pp, Qp, w):
    D = _Dev()
    Pp, Qp = np.ascontiguousarray(Pp, np.int32), np.ascontiguousarray(Qp, np.int32)
    n = len(Pp)
    if len(Qp) != n:
        raise ValueError("near: P and Q must have the same length")
    Ne, Nt = len(g['ep']), len(g['lt'])
    if n and (min(Pp.min(), Qp.min()) < 0 or max(Pp.max(), Qp.max()) >= Nt):
        raise ValueError("near: triangle index out of range")
    m, t, qd = D.mesh(g), D.tables(tb), D.quad(q)
    stat, ready = q.get('stat'), bool(q.get('stat_ready', False))
    if stat is not None and (not isinstance(stat, np.ndarray) or stat.dtype != np.float64 or
                             not stat.flags.c_contiguous or stat.size != 12 * n):
        raise ValueError("quad['stat']: a C-ordered float64 array of n x 12")
    d_stat = None
    if stat is not None:
        d_stat = D.put(stat, np.float64) if ready else torch.zeros(max(1, 12 * n), dtype=torch.float64,
                                                                    device='cuda')
    qc = torch.zeros(max(n, 1), dtype=torch.complex128, device='cuda')
    out = {}
    if mode == 0:
        Zd = D.put(Z[:Ne, :Ne], Z.dtype)
        check(lib().m25_near(0, P(Zd), c_long(Ne), c_int(Z.dtype == np.complex64), None, None, None, P(qc),
                             P(d_stat), c_int(ready), ctypes.byref(m), ctypes.byref(t), ctypes.byref(qd),
                             P(D.put(Pp, np.int32)), P(D.put(Qp, np.int32)), c_long(n), c_double(w), stream_ptr()),
              'near_into_dense')
        out['Z'] = Zd
    else:
        ri = torch.empty(max(9 * n, 1), dtype=torch.int32, device='cuda')
        ci = torch.empty_like(ri)
        vv = torch.empty(max(9 * n, 1), dtype=torch.complex128, device='cuda')
        check(lib().m25_near(2, None, c_long(0), 0, P(ri), P(ci), P(vv), P(qc), P(d_stat), c_int(ready),
                             ctypes.byref(m), ctypes.byref(t), ctypes.byref(qd), P(D.put(Pp, np.int32)),
                             P(D.put(Qp, np.int32)), c_long(n), c_double(w), stream_ptr()), 'near_coo')
        out.update(ri=ri[:9 * n], ci=ci[:9 * n], vv=vv[:9 * n])
    _done('near')
    if stat is not None and not ready:
        stat.reshape(-1)[:] = d_stat[:12 * n].cpu().numpy()
    out['qc'] = qc[:n]
    return out


def near_into_dense(Z, g, tb, q, P_, Q_, w):
    """Near-pair corrections added into Z[:Ne, :Ne]; returns the pairs' G_q corrections qcorr complex128[n]
    (mom25d_core.cpp:417-537). q['stat'] (n x 12, optional) keeps the analytic parts across frequencies:
    written when q['stat_ready'] is false, read when it is true."""
    _z_matrix(Z, len(g['ep']))
    Ne = len(g['ep'])
    o = _near(0, Z, g, tb, q, P_, Q_, w)
    Z[:Ne, :Ne] = o['Z'].cpu().numpy()
    return o['qc'].cpu().numpy()


def near_coo(g, tb, q, P_, Q_, w):
    """The near corrections as COO triplets (9 a pair, ri = -1 where unused): (ri, ci, vv, qcorr)
    (mom25d_core.cpp:559-575)."""
    o = _near(2, None, g, tb, q, P_, Q_, w)
    return o['ri'].cpu().numpy(), o['ci'].cpu().numpy(), o['vv'].cpu().numpy(), o['qc'].cpu().numpy()


def near_matvec(x, g, tb, q, P_, Q_, w):
    """y = dZ_near x for one column x complex128[Ne] (mom25d_core.cpp:540-556)."""
    Ne = len(g['ep'])
    x = np.ascontiguousarray(x, np.complex128).reshape(-1)
    if len(x) != Ne:
        raise ValueError(f"near_matvec: x must have {Ne} entries")
    o = _near(2, None, g, tb, q, P_, Q_, w)
    Xd = _lib.dev(x.reshape(Ne, 1), np.complex128)
    Y = torch.zeros_like(Xd)
    nnz = o['ri'].numel()
    if nnz:
        check(lib().m25_coo_spmm(P(o['ri']), P(o['ci']), P(o['vv']), c_long(nnz), P(Xd), 1, P(Y), stream_ptr()),
              'near_matvec')
    _done('near_matvec')
    return Y[:, 0].cpu().numpy()


def near_q(g, tb, q, P_, Q_, w):
    """The near pairs' G_q moment corrections alone, complex128[n] (mom25d_core.cpp:579)."""
    return _near(2, None, g, tb, q, P_, Q_, w)['qc'].cpu().numpy()


def near_pairs(cent, size, z, fac):
    """Near triangle pairs rho^2 + dz^2 < (fac max(size_p, size_q))^2, both orders, sorted by (p, q):
    (P, Q) int64 (mom25d_core.cpp:1216-1263)."""
    D = _Dev()
    cent = np.ascontiguousarray(cent, np.float64)
    size, z = np.ascontiguousarray(size, np.float64), np.ascontiguousarray(z, np.float64)
    Nt = len(size)
    if cent.shape != (Nt, 2) or z.shape != (Nt,):
        raise ValueError("near_pairs: cent (Nt, 2), size (Nt,), z (Nt,)")
    dc, ds, dz = D.put(cent, np.float64), D.put(size, np.float64), D.put(z, np.float64)
    off = torch.zeros(Nt + 1, dtype=torch.int64, device='cuda')
    total = ctypes.c_longlong(0)
    check(lib().m25_near_pairs(P(dc), P(ds), P(dz), c_int(Nt), c_double(fac), P(off), ctypes.byref(total), None,
                               None, stream_ptr()), 'near_pairs')
    n = total.value
    Pp = torch.empty(max(n, 1), dtype=torch.int32, device='cuda')
    Qp = torch.empty_like(Pp)
    check(lib().m25_near_pairs(P(dc), P(ds), P(dz), c_int(Nt), c_double(fac), P(off), ctypes.byref(total), P(Pp),
                               P(Qp), stream_ptr()), 'near_pairs')
    _done('near_pairs')
    return Pp[:n].cpu().numpy().astype(np.int64), Qp[:n].cpu().numpy().astype(np.int64)


# ---- via and table helpers ---------------------------------------------------------------------------------------
def radial_table_sum(px, py, W, vx, vy, table, dr):
    """out[t, v] = sum_q D(|P[t, q] - V[v]|) W[t, q] for a radial table D of step dr: complex128 (nt, nv)
    (mom25d_core.cpp:1269-1298)."""
    D = _Dev()
    px, py, W = (np.ascontiguousarray(a, np.float64) for a in (px, py, W))
    vx, vy = np.ascontiguousarray(vx, np.float64), np.ascontiguousarray(vy, np.float64)
    table = np.ascontiguousarray(table, np.complex128)
    if px.ndim != 2 or py.shape != px.shape or W.shape != px.shape or vx.shape != vy.shape:
        raise ValueError("radial_table_sum: px, py, W (nt, nq); vx, vy (nv,)")
    if len(table) < 2:
        raise ValueError("radial_table_sum: a table of at least 2 samples")
    nt, nq = px.shape
    out = torch.zeros((nt, len(vx)), dtype=torch.complex128, device='cuda')
    if nt and len(vx):
        check(lib().m25_radial_table_sum(P(D.put(px, np.float64)), P(D.put(py, np.float64)), P(D.put(W, np.float64)),
                                         c_long(nt), c_int(nq), P(D.put(vx, np.float64)), P(D.put(vy, np.float64)),
                                         c_int(len(vx)), P(D.put(table, np.complex128)), c_long(len(table)),
                                         c_double(dr), P(out), stream_ptr()), 'radial_table_sum')
    _done('radial_table_sum')
    return out.cpu().numpy()


def fan_q(g, tb, F):
    """G_q moments between every triangle and the fan triangles F: complex128 (Nt, len(F))
    (mom25d_core.cpp:1585-1603)."""
    D = _Dev()
    F = np.ascontiguousarray(F, np.int32)
    Nt = len(g['lt'])
    if F.size and (F.min() < 0 or F.max() >= Nt):
        raise ValueError("fan_q: triangle index out of range")
    m, t = D.mesh(g), D.tables(tb)
    out = torch.zeros((Nt, len(F)), dtype=torch.complex128, device='cuda')
    if len(F):
        check(lib().m25_fan_q(P(D.put(F, np.int32)), c_int(len(F)), P(out), ctypes.byref(m), ctypes.byref(t),
                              stream_ptr()), 'fan_q')
    _done('fan_q')
    return out.cpu().numpy()


def hankel_real(rho, kr, W):
    """sum_k J0(rho_i kr_k) W[s, k] over real kr: complex128 (nspec, len(rho)) (mom25d_core.cpp:1430-1454)."""
    D = _Dev()
    rho, kr = np.ascontiguousarray(rho, np.float64).reshape(-1), np.ascontiguousarray(kr, np.float64).reshape(-1)
    W = np.ascontiguousarray(np.atleast_2d(W), np.complex128)
    if W.shape[1] != len(kr):
        raise ValueError("hankel_real: W must be (nspec, len(kr))")
    out = torch.zeros((W.shape[0], len(rho)), dtype=torch.complex128, device='cuda')
    d_rho, d_kr = D.put(rho, np.float64), D.put(kr, np.float64)
    for s0 in range(0, W.shape[0], 16):
        Ws = D.put(W[s0:s0 + 16], np.complex128)
        ns = Ws.shape[0]
        if len(rho):
            check(lib().m25_hankel_real(P(d_rho), c_int(len(rho)), P(d_kr), c_int(len(kr)), P(Ws), c_int(ns),
                                        P(out[s0:s0 + ns]), stream_ptr()), 'hankel_real')
    _done('hankel_real')
    return out.cpu().numpy()


def bessel_jn_complex(n, z):
    """J_n(z) elementwise for complex z of any shape, n = 0, 1, 2 (mom25d_core.cpp:1510-1558)."""
    if n not in (0, 1, 2):
        raise ValueError("bessel_jn_complex: order 0, 1 or 2")
    D = _Dev()
    z = np.asarray(z, np.complex128)
    zd = D.put(z.reshape(-1), np.complex128)
    out = torch.empty_like(zd)
    if z.size:
        check(lib().m25_bessel_jn_complex(c_int(n), P(zd), c_long(z.size), P(out), stream_ptr()),
              'bessel_jn_complex')
    _done('bessel_jn_complex')
    return out.cpu().numpy().reshape(z.shape)


def scale_c64(Z, d):
    """Z <- diag(d) Z diag(d) in place (complex128, square) and its complex64 copy, returned
    (mom25d_core.cpp:1563-1580)."""
    if not isinstance(Z, np.ndarray) or Z.dtype != np.complex128 or not Z.flags.c_contiguous or Z.ndim != 2 \
            or Z.shape[0] != Z.shape[1]:
        raise ValueError("scale_c64: Z must be a square C-contiguous complex128 array")
    n = Z.shape[0]
    d = np.ascontiguousarray(d, np.float64)
    if d.shape != (n,):
        raise ValueError(f"scale_c64: d must have {n} entries")
    D = _Dev()
    Zd = D.put(Z, np.complex128)
    Zf = torch.empty((n, n), dtype=torch.complex64, device='cuda')
    check(lib().m25_equilibrate(P(Zd), c_long(n), c_long(n), P(D.put(d, np.float64)), None, P(Zf), stream_ptr()),
          'scale_c64')
    _done('scale_c64')
    Z[:] = Zd.cpu().numpy()
    return Zf.cpu().numpy()


def num_threads():
    """The host threads the reference's core would use; the kernels here run on the GPU."""
    return len(os.sched_getaffinity(0))
