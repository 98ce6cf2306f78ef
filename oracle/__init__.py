"""
oracle - TEST INFRASTRUCTURE ONLY. A CPU restatement of the reference's (lowprocess/mom25d) hot path, used as the
checker of the CUDA implementation by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference leg.
The product (mom25d_b200) never imports, links or runs anything here.

  oracle.c     the compiled core's kernels (mom25d_core.cpp) in plain C + OpenMP, built by build() into
               oracle/_build/liboracle.so; wrapped below with the reference core's own Python signatures
               (fill_far, near_into_dense, near_coo, ...), so the same dictionaries drive both
  green.py     the layered-media Green tables (multilayer.py, via.py: contour, Hankel transform, spline)
  via.py       the via kernels and via blocks (via.py, sim.py:_via_blocks)
  solve.py     equilibration, LAPACK LU (SciPy, the reference's own call), batched GMRES, the direct solve
  build_ref.sh the reference's own compiled core built from its sources into oracle/_ref/ (a second checker
               and the timed CPU baseline)

Pinning: tests/test_oracle.py checks this restatement against oracle/_ref (the reference's compiled core) and
against tests/golden/ fixtures generated by importing the reference (tests/golden/make_golden.py).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, '_build', 'liboracle.so')
_lib = None


def build(force=False):
    """Compile oracle.c (gcc -O3 -fopenmp, no FMA contraction: the reference core's own arithmetic)."""
    src = os.path.join(HERE, 'oracle.c')
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(src):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    subprocess.check_call(['gcc', '-O3', '-ffp-contract=off', '-fopenmp', '-shared', '-fPIC', '-std=gnu11', src,
                           '-o', LIB, '-lm'])
    return LIB


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
    return _lib


class _Tables(ctypes.Structure):
    _fields_ = [('ntab', ctypes.c_int), ('nfine', ctypes.c_int), ('L', ctypes.c_int)] + \
               [(n, ctypes.c_void_p) for n in ('A', 'Q', 'cA', 'cq', 'cAi', 'cqi', 'dr', 'd', 'dimg', 'tab', 'kind')]


class _Mesh(ctypes.Structure):
    _fields_ = [('Ne', ctypes.c_int), ('Nt', ctypes.c_int)] + \
               [(n, ctypes.c_void_p) for n in ('ep', 'em', 'lt', 'te', 'ap', 'am', 'vp', 'vm', 'cent', 'area',
                                               'ta', 'tv')]


def _c(a, dt):
    return np.ascontiguousarray(a, dt)


class _Hold:
    """Keeps the contiguous copies alive for the duration of a call."""
    def __init__(self):
        self.keep = []

    def ptr(self, a, dt):
        a = _c(a, dt)
        self.keep.append(a)
        return a.ctypes.data


def _mesh(g, h):
    m = _Mesh()
    m.Ne, m.Nt = len(g['ep']), len(g['lt'])
    for n in ('ep', 'em', 'lt', 'te'):
        setattr(m, n, h.ptr(g[n], np.int32))
    for n in ('ap', 'am', 'vp', 'vm', 'cent', 'area', 'ta', 'tv'):
        setattr(m, n, h.ptr(g[n], np.float64))
    return m


def _tables(tb, h):
    t = _Tables()
    A = _c(tb['A'], np.complex128)
    t.ntab, t.nfine, t.L = A.shape[0], A.shape[1], len(tb['tab'])
    for n in ('A', 'Q', 'cA', 'cq', 'cAi', 'cqi'):
        setattr(t, n, h.ptr(tb[n], np.complex128))
    for n in ('dr', 'd', 'dimg'):
        setattr(t, n, h.ptr(tb[n], np.float64))
    for n in ('tab', 'kind'):
        setattr(t, n, h.ptr(tb[n], np.int32))
    return t


# ---- the reference core's signatures (mom25d_core.cpp:1658-1702) ----------------------------------------------------
def fill_far(Z, g, tb, w):
    h = _Hold()
    assert Z.flags.c_contiguous and Z.dtype in (np.complex128, np.complex64)
    lib().orc_fill_far(ctypes.c_void_p(Z.ctypes.data), ctypes.c_size_t(Z.shape[1]),
                       ctypes.c_int(Z.dtype == np.complex64), ctypes.byref(_mesh(g, h)), ctypes.byref(_tables(tb, h)),
                       ctypes.c_double(w))


def fill_far_c64(Z, g, tb, w):
    fill_far(Z, g, tb, w)


def far_block(rows, cols, g, tb, w):
    h = _Hold()
    rows, cols = _c(rows, np.int32), _c(cols, np.int32)
    out = np.zeros((len(rows), len(cols)), complex)
    lib().orc_far_block(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(rows.ctypes.data), ctypes.c_int(len(rows)),
                        ctypes.c_void_p(cols.ctypes.data), ctypes.c_int(len(cols)), ctypes.byref(_mesh(g, h)),
                        ctypes.byref(_tables(tb, h)), ctypes.c_double(w))
    return out


def matvec_far_multi(X, g, tb, w):
    h = _Hold()
    X = _c(X, np.complex128)
    Y = np.zeros_like(X)
    lib().orc_matvec_far_multi(ctypes.c_void_p(Y.ctypes.data), ctypes.c_void_p(X.ctypes.data), ctypes.c_int(X.shape[1]),
                               ctypes.byref(_mesh(g, h)), ctypes.byref(_tables(tb, h)), ctypes.c_double(w))
    return Y


def _near(mode, Z, g, tb, q, P, Q, w, x=None):
    h = _Hold()
    P, Q = _c(P, np.int32), _c(Q, np.int32)
    n = len(P)
    qc = np.zeros(n, complex)
    ri = ci = vv = y = None
    if mode == 2:
        ri, ci, vv = np.zeros(9 * n, np.int32), np.zeros(9 * n, np.int32), np.zeros(9 * n, complex)
    if mode == 1:
        x = _c(x, np.complex128)
        y = np.zeros(len(g['ep']), complex)
    stat = q.get('stat')
    if stat is not None:
        assert stat.dtype == np.float64 and stat.flags.c_contiguous and stat.size == 12 * n
    vp = lambda a: ctypes.c_void_p(None if a is None else a.ctypes.data)
    lib().orc_near(ctypes.c_int(mode), vp(Z), ctypes.c_size_t(0 if Z is None else Z.shape[1]),
                   ctypes.c_int(Z is not None and Z.dtype == np.complex64), vp(ri), vp(ci), vp(vv), vp(x), vp(y),
                   vp(qc), vp(stat), ctypes.c_int(bool(q.get('stat_ready', False))), ctypes.byref(_mesh(g, h)),
                   ctypes.byref(_tables(tb, h)), ctypes.c_void_p(h.ptr(q['nodes'], np.float64)),
                   ctypes.c_void_p(h.ptr(q['tris'], np.int32)), ctypes.c_void_p(h.ptr(q['P3'], np.float64)),
                   ctypes.c_void_p(h.ptr(q['W3'], np.float64)), ctypes.c_void_p(h.ptr(q['P6'], np.float64)),
                   ctypes.c_void_p(h.ptr(q['W6'], np.float64)), vp(P), vp(Q), ctypes.c_int(n), ctypes.c_double(w))
    return qc, ri, ci, vv, y


def near_into_dense(Z, g, tb, q, P, Q, w):
    assert Z.flags.c_contiguous
    return _near(0, Z, g, tb, q, P, Q, w)[0]


def near_coo(g, tb, q, P, Q, w):
    qc, ri, ci, vv, _ = _near(2, None, g, tb, q, P, Q, w)
    return ri, ci, vv, qc


def near_matvec(x, g, tb, q, P, Q, w):
    return _near(1, None, g, tb, q, P, Q, w, x=x)[4]


def near_pairs(cent, size, z, fac):
    cent, size, z = _c(cent, np.float64), _c(size, np.float64), _c(z, np.float64)
    Nt = len(size)
    counts = np.zeros(Nt, np.int64)
    L = lib()
    L.orc_near_pairs.restype = ctypes.c_int64
    vp = lambda a: ctypes.c_void_p(a.ctypes.data)
    n = L.orc_near_pairs(vp(cent), vp(size), vp(z), ctypes.c_int(Nt), ctypes.c_double(fac), None, None, vp(counts))
    P, Q = np.zeros(n, np.int64), np.zeros(n, np.int64)
    L.orc_near_pairs(vp(cent), vp(size), vp(z), ctypes.c_int(Nt), ctypes.c_double(fac), vp(P), vp(Q), vp(counts))
    return P, Q


def radial_table_sum(px, py, W, vx, vy, table, dr):
    px, py, W = _c(px, np.float64), _c(py, np.float64), _c(W, np.float64)
    vx, vy, table = _c(vx, np.float64), _c(vy, np.float64), _c(table, np.complex128)
    nt, nq = px.shape
    out = np.zeros((nt, len(vx)), complex)
    vp = lambda a: ctypes.c_void_p(a.ctypes.data)
    lib().orc_radial_table_sum(vp(out), vp(px), vp(py), vp(W), ctypes.c_int64(nt), ctypes.c_int64(nq), vp(vx), vp(vy),
                               ctypes.c_int64(len(vx)), vp(table), ctypes.c_int64(len(table)), ctypes.c_double(dr))
    return out


def fan_q(g, tb, F):
    h = _Hold()
    F = _c(F, np.int32)
    out = np.zeros((len(g['lt']), len(F)), complex)
    lib().orc_fan_q(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(F.ctypes.data), ctypes.c_int(len(F)),
                    ctypes.byref(_mesh(g, h)), ctypes.byref(_tables(tb, h)))
    return out


def hankel_real(rho, kr, W):
    rho, kr, W = _c(rho, np.float64), _c(kr, np.float64), _c(np.atleast_2d(W), np.complex128)
    out = np.zeros((W.shape[0], len(rho)), complex)
    vp = lambda a: ctypes.c_void_p(a.ctypes.data)
    lib().orc_hankel_real(vp(out), vp(rho), ctypes.c_int(len(rho)), vp(kr), ctypes.c_int(len(kr)), vp(W),
                          ctypes.c_int(W.shape[0]))
    return out


def bessel_jn_complex(n, z):
    z = _c(z, np.complex128)
    out = np.zeros(z.shape, complex)
    lib().orc_bessel_jn_complex(ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(z.ctypes.data),
                                ctypes.c_int64(z.size), ctypes.c_int(n))
    return out


def scale_c64(Z, d):
    assert Z.flags.c_contiguous and Z.dtype == np.complex128
    d = _c(d, np.float64)
    out = np.zeros(Z.shape, np.complex64)
    lib().orc_scale_c64(ctypes.c_void_p(Z.ctypes.data), ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(d.ctypes.data),
                        ctypes.c_int64(Z.shape[0]))
    return out


def num_threads():
    return os.cpu_count() or 1
