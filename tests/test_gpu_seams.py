"""The two drop-in seams on the GPU: mom25d_b200.core (the reference's `_core` module, mom25d_core.cpp:1658-1702)
and mom25d_b200.backend.CudaBackend (the GPU LU backend, gpu.py:28-110), each against the oracle (the CPU
restatement pinned to the reference) on the same host arrays, the way the reference's own tests compare its core
with NumPy (test_solver.py:464-501, 584-639: 1e-12) and its GPU LU with LAPACK (test_gpu.py:210-235)."""
import importlib.util
import os

import numpy as np
import pytest
import scipy.linalg as sla

import oracle
from oracle import solve as osolve

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.fixture(scope='module')
def case():
    from mom25d_b200 import board as B, geometry as G
    spec = importlib.util.spec_from_file_location('mg', os.path.join(os.path.dirname(__file__), 'golden',
                                                                     'make_golden.py'))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    geo = G.Geometry(mg.small_board(B))
    od = osolve.Direct(geo)
    od.setup(3e9)
    return geo, od


def test_core_fill_far(case):
    from mom25d_b200 import core
    geo, od = case
    N, Ne, w = geo.N, geo.Ne, od.w
    Z = np.full((N, N), 7 + 1j)                                  # the via border must stay untouched
    core.fill_far(Z, geo.g, od.tb, w)
    Zo = np.full((N, N), 7 + 1j)
    oracle.fill_far(Zo, geo.g, od.tb, w)
    assert rel(Z, Zo) < 1e-13
    assert np.all(Z[Ne:, :] == 7 + 1j) and np.all(Z[:, Ne:] == 7 + 1j)
    Z64 = np.zeros((N, N), np.complex64)
    core.fill_far_c64(Z64, geo.g, od.tb, w)
    ref = Zo[:Ne, :Ne].astype(np.complex64)
    assert np.abs(Z64[:Ne, :Ne] - ref).max() <= 2 ** -22 * np.abs(ref).max()
    rows, cols = np.arange(0, Ne, 7, dtype=np.int32), np.arange(3, Ne, 5, dtype=np.int32)
    assert rel(core.far_block(rows, cols, geo.g, od.tb, w), oracle.far_block(rows, cols, geo.g, od.tb, w)) < 1e-13
    X = np.random.default_rng(0).normal(size=(Ne, 2)) + 1j
    assert rel(core.matvec_far_multi(X, geo.g, od.tb, w), oracle.matvec_far_multi(X, geo.g, od.tb, w)) < 1e-12
    assert rel(core.matvec_far(X[:, 0], geo.g, od.tb, w), oracle.matvec_far_multi(X, geo.g, od.tb, w)[:, 0]) < 1e-12


def test_core_near_and_its_kept_analytic_parts(case):
    from mom25d_b200 import core
    geo, od = case
    Ne, w = geo.Ne, od.w
    n = len(od.nP32)
    q = dict(geo.q, stat=np.zeros((n, 12)), stat_ready=False)
    qo = dict(geo.q, stat=np.zeros((n, 12)), stat_ready=False)
    Z0 = np.zeros((Ne, Ne), complex)
    oracle.fill_far(Z0, geo.g, od.tb, w)
    for ready in (False, True):
        q['stat_ready'] = qo['stat_ready'] = ready
        Z, Zo = Z0.copy(), Z0.copy()
        qc = core.near_into_dense(Z, geo.g, od.tb, q, od.nP32, od.nQ32, w)
        qco = oracle.near_into_dense(Zo, geo.g, od.tb, qo, od.nP32, od.nQ32, w)
        assert rel(Z, Zo) < 1e-12 and rel(qc, qco) < 1e-12
        assert np.abs(q['stat'] - qo['stat']).max() <= 1e-12 * np.abs(qo['stat']).max()
    ri, ci, vv, qc = core.near_coo(geo.g, od.tb, geo.q, od.nP32, od.nQ32, w)
    r1, c1, v1, q1 = oracle.near_coo(geo.g, od.tb, geo.q, od.nP32, od.nQ32, w)
    assert np.array_equal(ri, r1)
    ok = r1 >= 0
    assert np.array_equal(ci[ok], c1[ok]) and rel(vv[ok], v1[ok]) < 1e-12 and rel(qc, q1) < 1e-12
    x = np.random.default_rng(1).normal(size=Ne) + 0.5j
    assert rel(core.near_matvec(x, geo.g, od.tb, geo.q, od.nP32, od.nQ32, w),
               oracle.near_matvec(x, geo.g, od.tb, geo.q, od.nP32, od.nQ32, w)) < 1e-12
    assert rel(core.near_q(geo.g, od.tb, geo.q, od.nP32, od.nQ32, w), q1) < 1e-12
    P, Q = core.near_pairs(geo.g['cent'], geo.tri_size, geo.tri_z, geo.near_fac)
    assert P.dtype == np.int64 and np.array_equal(P, od.nP) and np.array_equal(Q, od.nQ)


def test_core_via_and_table_helpers(case, golden):
    from mom25d_b200 import core
    geo, od = case
    F = np.arange(0, geo.Nt, 9, dtype=np.int32)
    assert rel(core.fan_q(geo.g, od.tb, F), oracle.fan_q(geo.g, od.tb, F)) < 1e-12
    rng = np.random.default_rng(2)
    px, py, W = rng.uniform(-2e-3, 2e-3, (40, 6)), rng.uniform(-2e-3, 2e-3, (40, 6)), rng.uniform(0, 1, (40, 6))
    vx, vy = rng.uniform(-2e-3, 2e-3, 5), rng.uniform(-2e-3, 2e-3, 5)
    table = rng.normal(size=300) + 1j * rng.normal(size=300)
    assert rel(core.radial_table_sum(px, py, W, vx, vy, table, 2e-5),
               oracle.radial_table_sum(px, py, W, vx, vy, table, 2e-5)) < 1e-13
    rho, kr = np.linspace(0, 5e-3, 37), np.linspace(10, 4e4, 500)
    Wh = rng.normal(size=(3, 500)) + 1j * rng.normal(size=(3, 500))
    # CUDA's j0 against glibc's, summed over 500 terms of random sign: the reference's core-vs-SciPy bar, 1e-12
    assert rel(core.hankel_real(rho, kr, Wh), oracle.hankel_real(rho, kr, Wh)) < 1e-12
    for n in range(3):
        assert np.abs(core.bessel_jn_complex(n, golden['jn_z']) - golden['jn_%d' % n]).max() <= \
            1e-13 * np.abs(golden['jn_%d' % n]).max()
    Z = rng.normal(size=(60, 60)) + 1j * rng.normal(size=(60, 60))
    d = rng.uniform(0.5, 2, 60)
    Zo = Z.copy()
    c64 = core.scale_c64(Z, d)
    c64o = oracle.scale_c64(Zo, d)
    assert rel(Z, Zo) < 1e-15 and np.array_equal(c64, c64o)
    with pytest.raises(ValueError):
        core.scale_c64(Z.astype(np.complex64), d)


@pytest.mark.parametrize('dt', [np.complex64, np.complex128])
def test_backend_factor_solve_download(dt):
    """The reference's LU test (test_gpu.py:210-235): N = 300, + 4 sqrt(N) I, rows 0 and 7 interchanged; pivots
    equal to LAPACK's, the factor to round-off, solves of Z X = R."""
    from mom25d_b200.backend import CudaBackend
    n = 300
    rng = np.random.default_rng(4)
    Z = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 4 * np.sqrt(n) * np.eye(n)).astype(dt)
    Z[[0, 7]] = Z[[7, 0]]
    be = CudaBackend()
    assert be.fits(n) and be.mem_total() > be.mem_free() > 0
    be.factor(np.ascontiguousarray(Z))
    lu, piv = be.download()
    lu_ref, piv_ref = sla.lu_factor(Z.T.astype(complex))
    assert np.array_equal(piv, piv_ref)
    tol = 1e-4 if dt == np.complex64 else 1e-12
    assert np.abs(lu - lu_ref).max() < tol * np.abs(lu_ref).max()
    R = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
    X = be.solve(R)
    assert X.dtype == np.complex128 and X.shape == (n, 2)
    x = np.linalg.solve(Z.astype(complex), R)
    assert np.abs(X - x).max() < (1e-4 if dt == np.complex64 else 1e-11) * np.abs(x).max()
    assert np.allclose(be.solve(R[:, 0]), X[:, 0], rtol=0, atol=1e-5 * np.abs(x).max())
    be.release()
    with pytest.raises(RuntimeError):
        be.solve(R)


@pytest.mark.parametrize('dt', [np.complex64, np.complex128])
def test_backend_pivoting_over_many_outer_panels(dt):
    """A Gaussian matrix without a diagonal boost (row interchanges in nearly every column) over a dozen outer
    panels of 256 columns, so that the interchanges of each panel meet the trailing update of the previous one
    that runs beside it: the solve's backward error ||Z x - r|| / (||Z|| ||x||) at the factor's round-off."""
    from mom25d_b200.backend import CudaBackend
    n = 3000
    rng = np.random.default_rng(21)
    Z = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(dt)
    be = CudaBackend()
    be.factor(np.ascontiguousarray(Z))
    _, piv = be.download()
    assert np.count_nonzero(piv != np.arange(n)) > n // 2
    R = rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3))
    X = be.solve(R)
    Zc = Z.astype(complex)
    berr = np.linalg.norm(Zc @ X - R) / (np.linalg.norm(Zc) * np.linalg.norm(X))
    assert berr < (5e-6 if dt == np.complex64 else 1e-14), berr     # LAPACK in complex64: 8.6e-7
    be.release()


@pytest.mark.parametrize('dt', [np.complex64, np.complex128])
def test_lookahead_factor_equals_the_in_order_one(dt, monkeypatch):
    """The look-ahead LU (the next outer panel factored while the rest of the previous trailing update runs on a
    second stream) gives the same bits as the same steps on one stream (M25_LOOKAHEAD=0): no step reads what the
    other stream writes."""
    from mom25d_b200.backend import CudaBackend
    n = 2000
    rng = np.random.default_rng(22)
    Z = np.ascontiguousarray((rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(dt))
    out = []
    for la in ('1', '0', '1'):
        monkeypatch.setenv('M25_LOOKAHEAD', la)
        be = CudaBackend()
        be.factor(Z)
        out.append(be.download())
        be.release()
    for lu, piv in out[1:]:
        assert np.array_equal(piv, out[0][1]) and np.array_equal(lu, out[0][0])
