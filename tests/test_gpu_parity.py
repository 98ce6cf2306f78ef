"""Parity of the CUDA hot path with the oracle (a CPU restatement of the reference, pinned in test_oracle.py) and
with the golden fixtures the reference itself wrote. All through the C ABI (libmom25d_b200.so)."""
import ctypes
import importlib.util
import os

import numpy as np
import pytest
import scipy.linalg as sla

import oracle
from oracle import green, solve as osolve

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')


def _small_board():
    from mom25d_b200 import board as B
    spec = importlib.util.spec_from_file_location('mg', os.path.join(os.path.dirname(__file__), 'golden',
                                                                     'make_golden.py'))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg.small_board(B)


@pytest.fixture(scope='module')
def small():
    from mom25d_b200 import geometry as G
    from mom25d_b200.operator import DirectSolver
    geo = G.Geometry(_small_board())
    return geo, DirectSolver(geo), osolve.Direct(geo)


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def upload_tables(tb):
    """The oracle's tb dictionary as device tables (the kernels alone, without the table builder)."""
    from mom25d_b200 import _lib
    d = {k: _lib.dev(tb[k], np.int32 if k in ('tab', 'kind') else (np.float64 if k in ('dr', 'd', 'dimg') else
                                                                    np.complex128)) for k in tb}
    T = _lib.Tables(tb['A'].shape[0], tb['A'].shape[1], len(tb['tab']),
                    *[_lib.P(d[k]) for k in ('A', 'Q', 'cA', 'cq', 'cAi', 'cqi', 'dr', 'd', 'dimg', 'tab', 'kind')])
    return T, d


def test_near_pairs_match(small):
    geo, ds, od = small
    n = ds.dg.npairs
    assert np.array_equal(ds.dg.nP[:n].cpu().numpy(), od.nP) and np.array_equal(ds.dg.nQ[:n].cpu().numpy(), od.nQ)


@pytest.mark.parametrize('f', [0.5e9, 3.0e9, 10e9])
def test_green_tables_match(small, f):
    from mom25d_b200.device import DeviceTables
    geo, ds, od = small
    od.setup(f)
    dt = DeviceTables(ds.dg, f, single=True)
    hd = dt.host_dict(geo)
    # The image coefficients come from the network's large-kr limit times exp(18) (multilayer.py:279-285): their
    # last digits depend on the libm in use, and the tables absorb the difference. What the fill uses is the total
    # kernel A_rest + sum c / sqrt(rho^2 + d^2): that is compared (at rho > 0), and the coefficients loosely.
    rho = np.linspace(0, geo.rho_max, 8192)[1:]
    for t in range(len(hd['kind'])):
        for k, c, ci in (('A', 'cA', 'cAi'), ('Q', 'cq', 'cqi')):
            tot = lambda h: (h[k][t][1:] + (h[c][t] / rho if h['kind'][t] == 0 else
                                             h[c][t] / np.hypot(rho, h['d'][t]) if h['kind'][t] == 1 else 0)
                             + (h[ci][t] / np.hypot(rho, h['dimg'][t]) if h['dimg'][t] > 0 else 0))
            assert rel(tot(hd), tot(od.tb)) < 1e-11, (t, k)
    for k in ('cA', 'cq', 'd', 'dimg', 'dr'):
        assert np.allclose(hd[k], od.tb[k], rtol=1e-12, atol=0), k
    for k in ('cAi', 'cqi'):
        assert np.allclose(hd[k], od.tb[k], rtol=1e-6, atol=0), k
    assert np.array_equal(hd['kind'], od.tb['kind'])
    # the mixed fill's complex64 tables: the same spline on the same grid, rounded
    A32 = dt.AQ32.cpu().numpy()
    n = len(hd['kind'])
    rho32 = np.linspace(0, geo.rho_max, A32.shape[1])
    from scipy.interpolate import CubicSpline
    H = dt.H.cpu().numpy()
    for i in range(n):
        want = CubicSpline(ds.dg.rho_coarse, H[i])(rho32)
        assert np.abs(A32[i] - want).max() <= 1e-6 * np.abs(want).max()


def test_fill_far_and_near_kernels_match_the_oracle(small):
    from mom25d_b200 import _lib
    geo, ds, od = small
    f = 3e9
    od.setup(f)
    T, keep = upload_tables(od.tb)
    Ne, w = geo.Ne, 2 * np.pi * f
    Z = torch.zeros((Ne, Ne), dtype=torch.complex128, device='cuda')
    _lib.check(_lib.lib().m25_fill_far(_lib.P(Z), ctypes.c_long(Ne), 0, ctypes.byref(ds.dg.mesh), ctypes.byref(T),
                                       None, ctypes.c_double(w), _lib.stream_ptr()))
    Zo = np.zeros((Ne, Ne), complex)
    oracle.fill_far(Zo, geo.g, od.tb, w)
    Zg = Z.cpu().numpy()
    assert rel(Zg, Zo) < 1e-13
    assert np.array_equal(Zg, Zg.T)                               # written symmetric, as the reference does
    qc = torch.zeros(ds.dg.npairs, dtype=torch.complex128, device='cuda')
    stat = torch.zeros(12 * ds.dg.npairs, dtype=torch.float64, device='cuda')
    for ready in (0, 1):                                          # computes, then reuses the analytic parts
        Zr = Z.clone()
        _lib.check(_lib.lib().m25_near(0, _lib.P(Zr), ctypes.c_long(Ne), 0, None, None, None, _lib.P(qc), _lib.P(stat),
                                       ready, ctypes.byref(ds.dg.mesh), ctypes.byref(T), ctypes.byref(ds.dg.quad),
                                       _lib.P(ds.dg.nP), _lib.P(ds.dg.nQ), ctypes.c_long(ds.dg.npairs),
                                       ctypes.c_double(w), _lib.stream_ptr()))
        _lib.sync_check()
        Zn = Zo.copy()
        qo = oracle.near_into_dense(Zn, geo.g, od.tb, geo.q, od.nP32, od.nQ32, w)
        assert rel(Zr.cpu().numpy(), Zn) < 1e-12
        assert rel(qc.cpu().numpy(), qo) < 1e-12
    # COO triplets
    n9 = 9 * ds.dg.npairs
    ri = torch.empty(n9, dtype=torch.int32, device='cuda'); ci = torch.empty_like(ri)
    vv = torch.empty(n9, dtype=torch.complex128, device='cuda')
    _lib.check(_lib.lib().m25_near(2, None, ctypes.c_long(0), 0, _lib.P(ri), _lib.P(ci), _lib.P(vv), _lib.P(qc),
                                   _lib.P(stat), 1, ctypes.byref(ds.dg.mesh), ctypes.byref(T), ctypes.byref(ds.dg.quad),
                                   _lib.P(ds.dg.nP), _lib.P(ds.dg.nQ), ctypes.c_long(ds.dg.npairs), ctypes.c_double(w),
                                   _lib.stream_ptr()))
    r1, c1, v1, _ = oracle.near_coo(geo.g, od.tb, geo.q, od.nP32, od.nQ32, w)
    rg = ri.cpu().numpy()
    assert np.array_equal(rg, r1)
    ok = r1 >= 0
    assert np.array_equal(ci.cpu().numpy()[ok], c1[ok])
    assert np.abs(vv.cpu().numpy()[ok] - v1[ok]).max() <= 1e-12 * np.abs(v1[ok]).max()
    # matrix-free far product
    X = np.random.default_rng(0).normal(size=(Ne, 3)) + 1j * np.random.default_rng(1).normal(size=(Ne, 3))
    Xd = _lib.dev(X, np.complex128)
    Yd = torch.empty_like(Xd)
    work = torch.empty(6 * geo.Nt * 3, dtype=torch.complex128, device='cuda')
    _lib.check(_lib.lib().m25_matvec_far_multi(_lib.P(Xd), 3, _lib.P(Yd), _lib.P(work), ctypes.byref(ds.dg.mesh),
                                               ctypes.byref(T), ctypes.c_double(w), _lib.stream_ptr()))
    Yo = oracle.matvec_far_multi(X, geo.g, od.tb, w)
    assert rel(Yd.cpu().numpy(), Yo) < 1e-12
    assert rel(Yo, Zo @ X) < 1e-12                               # (the product is the far field's)


def test_impedance_matches_the_reference(small, golden):
    geo, ds, od = small
    f = float(golden['board_f'][0])
    Z = ds.impedance(f, 'double').cpu().numpy()
    Zr = golden['board_Z']
    assert rel(Z, Zr) <= 1e-10                                    # the drop-in bar: Z to 1e-10 (Frobenius)
    Zo = od.impedance(f)
    assert rel(Z, Zo) <= 1e-10


def test_direct_solve_matches_the_reference(small, golden):
    geo, ds, od = small
    f = float(golden['board_f'][0])
    X = ds.solve_direct(f, geo.excitation(), precision='double').cpu().numpy()
    S = geo.sparams_from_currents(X)
    assert np.abs(S - golden['board_S_double']).max() <= 1e-8      # the drop-in bar: max |dS| 1e-8
    assert np.abs(X - golden['board_I_double']).max() <= 1e-8 * np.abs(golden['board_I_double']).max()


def test_mixed_solve_matches_the_reference(small, golden):
    geo, ds, od = small
    f = float(golden['board_f'][0])
    X = ds.solve_direct(f, geo.excitation(), precision='mixed').cpu().numpy()
    S = geo.sparams_from_currents(X)
    assert np.abs(S - golden['board_S_double']).max() <= 1e-4      # the mixed-precision bar
    assert np.abs(S - golden['board_S_double']).max() <= 1e-5      # (refined to 1e-6: well inside it)
    assert max(ds.iters) <= 30


def test_mixed_matrix_free_path_matches_the_reference(golden):
    """The mixed path without a resident double Z (complex64 fill, matrix-free double refinement operator)."""
    from mom25d_b200 import geometry as G
    from mom25d_b200.operator import DirectSolver
    geo = G.Geometry(_small_board())
    ds = DirectSolver(geo)
    ds.hybrid = False
    f = float(golden['board_f'][0])
    S = geo.sparams_from_currents(ds.solve_direct(f, geo.excitation(), precision='mixed').cpu().numpy())
    assert ds.last_path == 'mixed'
    assert np.abs(S - golden['board_S_double']).max() <= 1e-5


def test_mixed_with_a_kept_lu_matches_the_reference(golden):
    """A complex64 LU factored at 0.9 f preconditions the solve at f (fast.py:996-1084): no new factorisation,
    the same S to the mixed bar."""
    from mom25d_b200 import geometry as G
    from mom25d_b200.operator import DirectSolver
    geo = G.Geometry(_small_board())
    ds = DirectSolver(geo)
    f = float(golden['board_f'][0])
    ds.solve_direct(0.9 * f, geo.excitation(), precision='mixed')
    assert ds.last_path == 'fresh' and len(ds.kept) == 1
    X = ds.solve_direct(f, geo.excitation(), precision='mixed').cpu().numpy()
    assert ds.last_path == 'reused' and ds.last_lu_ms is None
    S = geo.sparams_from_currents(X)
    assert np.abs(S - golden['board_S_double']).max() <= 1e-5


@pytest.mark.parametrize('k', [1, 3, 8, 11, 16])
def test_dense_double_product(k):
    """The refinement's dense product Y = Z X (row-major Z, N x k X) against NumPy, ragged sizes."""
    from mom25d_b200 import _lib
    rng = np.random.default_rng(k)
    n = 1000 + 37 * k
    Z = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    X = rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k))
    Zd, Xd = _lib.dev(Z), _lib.dev(X)
    Yd = torch.empty_like(Xd)
    _lib.check(_lib.lib().m25_zgemm_skinny(_lib.P(Zd), ctypes.c_long(n), n, _lib.P(Xd), k, _lib.P(Yd),
                                           _lib.stream_ptr()))
    ref = Z @ X
    assert np.abs(Yd.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize('single,n', [(0, 300), (1, 300), (0, 1000), (1, 1000), (0, 3001)])
def test_lu_matches_lapack(single, n):
    """The LU against LAPACK (SciPy's lu_factor of Z^T): the same pivots, the factor to round-off, the solves
    (the reference's own LU test, test_gpu.py:210-235: N = 300, + 4 sqrt(N) I, rows 0 and 7 interchanged)."""
    from mom25d_b200 import _lib
    rng = np.random.default_rng(3)
    dt = np.complex64 if single else np.complex128
    Z = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(dt)
    Z += (4 * np.sqrt(n) * np.eye(n)).astype(dt)
    Z[[0, 7]] = Z[[7, 0]]
    Zd = _lib.dev(Z)
    ipiv = torch.empty(n, dtype=torch.int32, device='cuda')
    nb = int(_lib.lib().m25_getrf_workspace(n, single))
    work = torch.empty(nb, dtype=torch.uint8, device='cuda')
    _lib.check(_lib.lib().m25_getrf(_lib.P(Zd), ctypes.c_long(n), n, _lib.P(ipiv), single, 0, _lib.P(work),
                                    ctypes.c_size_t(nb), _lib.stream_ptr()))
    _lib.sync_check()
    lu_ref, piv_ref = sla.lu_factor(Z.T.astype(complex))
    lu = Zd.cpu().numpy().T                                         # the factor of Z^T (column-major in memory)
    assert np.array_equal(ipiv.cpu().numpy(), piv_ref)
    tol = 1e-4 if single else 1e-12
    assert np.abs(lu - lu_ref).max() < tol * np.abs(lu_ref).max()
    R = rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3))
    x = np.linalg.solve(Z.astype(complex), R)
    Rd = _lib.dev(R.astype(dt))
    _lib.check(_lib.lib().m25_getrs(_lib.P(Zd), ctypes.c_long(n), n, _lib.P(ipiv), single, _lib.P(Rd), 3,
                                    _lib.stream_ptr()))
    assert np.abs(Rd.cpu().numpy() - x).max() < (1e-4 if single else 1e-11) * np.abs(x).max()


@pytest.mark.parametrize('pattern', ['shift', 'reverse', 'random'])
@pytest.mark.parametrize('single,tf32', [(0, 0), (1, 0), (1, 1)])
def test_lu_row_interchange_patterns(pattern, single, tf32):
    """Row interchanges composed into one permutation per panel (the LU's interchange plans): matrices whose
    pivots are forced (Z^T = s P + noise, P a permutation: column j's pivot is the row P puts there), against
    LAPACK's pivots and factor. 'shift' (p_i = i + 1) makes every interchange chain to the one before it (the
    longest chains the plan resolves); 'reverse' moves rows far below the panel; N = 700: three outer panels, the
    last ragged, so the in-panel, look-ahead and far-column interchanges all run."""
    from mom25d_b200 import _lib
    n = 700
    rng = np.random.default_rng(7)
    sigma = {'shift': (np.arange(n) + 1) % n, 'reverse': np.arange(n)[::-1].copy(),
             'random': rng.permutation(n)}[pattern]
    dt = np.complex64 if single else np.complex128
    A = 0.1 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    A[sigma, np.arange(n)] += 10 * n * np.exp(1j * rng.uniform(0, 2 * np.pi, n))
    Z = np.ascontiguousarray(A.T).astype(dt)
    Zd = _lib.dev(Z)
    ipiv = torch.empty(n, dtype=torch.int32, device='cuda')
    nb = int(_lib.lib().m25_getrf_workspace(n, single))
    work = torch.empty(nb, dtype=torch.uint8, device='cuda')
    _lib.check(_lib.lib().m25_getrf(_lib.P(Zd), ctypes.c_long(n), n, _lib.P(ipiv), single, tf32, _lib.P(work),
                                    ctypes.c_size_t(nb), _lib.stream_ptr()))
    _lib.sync_check()
    lu_ref, piv_ref = sla.lu_factor(Z.T.astype(complex))
    assert np.count_nonzero(piv_ref != np.arange(n)) > n // 3
    assert np.array_equal(ipiv.cpu().numpy(), piv_ref)
    lu = Zd.cpu().numpy().T
    tol = 1e-5 if single else 1e-13
    assert np.abs(lu - lu_ref).max() < tol * np.abs(lu_ref).max()


def test_complex_bessel_matches_the_reference(golden):
    from mom25d_b200 import _lib
    z = _lib.dev(golden['jn_z'], np.complex128)
    out = torch.empty_like(z)
    for n in range(3):
        _lib.check(_lib.lib().m25_bessel_jn_complex(n, _lib.P(z), ctypes.c_long(z.numel()), _lib.P(out),
                                                    _lib.stream_ptr()))
        ref = golden['jn_%d' % n]
        assert np.abs(out.cpu().numpy() - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.parametrize('n', [700, 2000, 4100])
def test_lu_with_tensor_core_updates(n):
    """The complex64 LU with its trailing updates on the tensor cores (3xTF32): a factor as good as the FP32 one
    (backward error at single-precision level) and solves that match. 4100: 17 outer blocks, the last ragged, so
    every part of the two-stream schedule runs (the look-ahead columns, the far columns' first slice and rest)."""
    from mom25d_b200 import _lib
    rng = np.random.default_rng(5)
    Z = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))).astype(np.complex64)
    Z += (4 * np.sqrt(n) * np.eye(n)).astype(np.complex64)
    Zd = _lib.dev(Z)
    ipiv = torch.empty(n, dtype=torch.int32, device='cuda')
    nb = int(_lib.lib().m25_getrf_workspace(n, 1))
    work = torch.empty(nb, dtype=torch.uint8, device='cuda')
    _lib.check(_lib.lib().m25_getrf(_lib.P(Zd), ctypes.c_long(n), n, _lib.P(ipiv), 1, 1, _lib.P(work),
                                    ctypes.c_size_t(nb), _lib.stream_ptr()))
    _lib.sync_check()
    lu_ref, piv_ref = sla.lu_factor(Z.T.astype(complex))
    lu = Zd.cpu().numpy().T
    assert np.mean(ipiv.cpu().numpy() == piv_ref) > 0.99        # (rounding may move a near-tie)
    P = np.arange(n)
    for i, p in enumerate(ipiv.cpu().numpy()):
        P[[i, p]] = P[[p, i]]
    Lm, Um = np.tril(lu, -1) + np.eye(n), np.triu(lu)
    A = Z.T.astype(complex)
    assert np.abs(Lm @ Um - A[P]).max() < 1e-5 * np.abs(A).max()
    R = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
    x = np.linalg.solve(Z.astype(complex), R)
    Rd = _lib.dev(R.astype(np.complex64))
    _lib.check(_lib.lib().m25_getrs(_lib.P(Zd), ctypes.c_long(n), n, _lib.P(ipiv), 1, _lib.P(Rd), 2, _lib.stream_ptr()))
    assert np.abs(Rd.cpu().numpy() - x).max() < 1e-4 * np.abs(x).max()


@pytest.mark.parametrize('n,nrhs', [(9509, 3), (9600, 8), (19000, 16)])
def test_complex64_solves_over_several_blocks_a_cta(n, nrhs):
    """The complex64 solves where every CTA owns two or more 64-row blocks, odd and even n (16- and 8-byte
    copies of the factor tiles), 3 to 16 right-hand sides: against cuSOLVER's complex128 solve of the same Z."""
    from mom25d_b200 import _lib
    g = torch.Generator(device='cuda').manual_seed(n)
    Z = torch.complex(torch.randn(n, n, generator=g, device='cuda'), torch.randn(n, n, generator=g, device='cuda'))
    Z.diagonal().add_(4 * n ** 0.5)
    R = torch.complex(torch.randn(n, nrhs, generator=g, device='cuda'), torch.randn(n, nrhs, generator=g,
                                                                                     device='cuda'))
    x = torch.linalg.solve(Z.to(torch.complex128), R.to(torch.complex128))
    F = Z.clone()
    ipiv = torch.empty(n, dtype=torch.int32, device='cuda')
    nb = int(_lib.lib().m25_getrf_workspace(n, 1))
    work = torch.empty(nb, dtype=torch.uint8, device='cuda')
    _lib.check(_lib.lib().m25_getrf(_lib.P(F), ctypes.c_long(n), n, _lib.P(ipiv), 1, 1, _lib.P(work),
                                    ctypes.c_size_t(nb), _lib.stream_ptr()))
    for _ in range(2):                                               # twice: the flags' epochs
        X = R.clone()
        _lib.check(_lib.lib().m25_getrs(_lib.P(F), ctypes.c_long(n), n, _lib.P(ipiv), 1, _lib.P(X), nrhs,
                                        _lib.stream_ptr()))
        _lib.sync_check()
        err = (X.to(torch.complex128) - x).abs().max().item() / x.abs().max().item()
        assert err < 1e-4, err


@pytest.mark.parametrize('n,nrhs,single', [(2048, 8, 1), (2049, 1, 1), (2301, 5, 1), (5000, 8, 1), (18788, 8, 1),
                                           (2049, 3, 0), (5000, 8, 0)])
def test_solves_by_256_row_blocks(n, nrhs, single):
    """The solves by 256-row diagonal blocks (inverted once per factor, with their couplings to the two blocks
    solved before them: one product a block along the chain), complex64 and complex128: whole and ragged last blocks
    and chunks (2048, 2049: a last block of one row), odd n (8-byte copies of complex64 factor tiles), 1 to 8
    right-hand sides, a factor whose every column takes a row interchange; against the complex128 solve of the same
    Z, twice in a row (the flags' epochs)."""
    from mom25d_b200 import _lib
    L = _lib.lib()
    L.m25_getrs_aux_bytes.restype = ctypes.c_size_t
    rdt, cdt = (torch.float32, torch.complex64) if single else (torch.float64, torch.complex128)
    g = torch.Generator(device='cuda').manual_seed(n)
    sigma = torch.randperm(n, generator=g, device='cuda')
    A = 0.1 * torch.complex(torch.randn(n, n, generator=g, device='cuda', dtype=rdt),
                            torch.randn(n, n, generator=g, device='cuda', dtype=rdt))
    phase = 2 * np.pi * torch.rand(n, generator=g, device='cuda', dtype=rdt)
    A[sigma, torch.arange(n, device='cuda')] += 10 * n * torch.exp(1j * phase).to(cdt)
    Z = A.T.contiguous()
    R = torch.complex(torch.randn(n, nrhs, generator=g, device='cuda', dtype=rdt),
                      torch.randn(n, nrhs, generator=g, device='cuda', dtype=rdt))
    x = torch.linalg.solve(Z.to(torch.complex128), R.to(torch.complex128))
    F = Z.clone()
    ipiv = torch.empty(n, dtype=torch.int32, device='cuda')
    nb = int(L.m25_getrf_workspace(n, single))
    work = torch.empty(nb, dtype=torch.uint8, device='cuda')
    _lib.check(L.m25_getrf(_lib.P(F), ctypes.c_long(n), n, _lib.P(ipiv), single, single, _lib.P(work),
                           ctypes.c_size_t(nb), _lib.stream_ptr()))
    del work
    assert (ipiv.cpu().numpy() != np.arange(n)).mean() > 0.9
    na = int(L.m25_getrs_aux_bytes(n, single))
    aux = torch.empty(na, dtype=torch.uint8, device='cuda')
    _lib.check(L.m25_getrs_prepare(_lib.P(F), ctypes.c_long(n), n, _lib.P(ipiv), single, _lib.P(aux),
                                   ctypes.c_size_t(na), _lib.stream_ptr()), 'm25_getrs_prepare')
    for _ in range(2):
        X = R.clone()
        _lib.check(L.m25_getrs_aux(_lib.P(F), ctypes.c_long(n), n, single, _lib.P(aux), _lib.P(X), nrhs,
                                   _lib.stream_ptr()), 'm25_getrs_aux')
        _lib.sync_check()
        err = (X.to(torch.complex128) - x).abs().max().item() / x.abs().max().item()
        assert err < (1e-5 if single else 1e-12), err


@pytest.mark.parametrize('n,nrhs', [(9509, 1), (18788, 8), (19000, 16)])
def test_complex128_solves_over_several_blocks_a_cta(n, nrhs):
    """The complex128 solves through the same pipelined kernel (32-row factor tiles, one inverse buffer) where the
    CTAs own one and two 64-row blocks, 1 to 16 right-hand sides: against cuSOLVER's solve of the same Z, at double
    precision's bar."""
    from mom25d_b200 import _lib
    g = torch.Generator(device='cuda').manual_seed(n)
    Z = torch.complex(torch.randn(n, n, generator=g, device='cuda', dtype=torch.float64),
                      torch.randn(n, n, generator=g, device='cuda', dtype=torch.float64))
    Z.diagonal().add_(4 * n ** 0.5)
    R = torch.complex(torch.randn(n, nrhs, generator=g, device='cuda', dtype=torch.float64),
                      torch.randn(n, nrhs, generator=g, device='cuda', dtype=torch.float64))
    x = torch.linalg.solve(Z, R)
    F = Z.clone()
    ipiv = torch.empty(n, dtype=torch.int32, device='cuda')
    nb = int(_lib.lib().m25_getrf_workspace(n, 0))
    work = torch.empty(nb, dtype=torch.uint8, device='cuda')
    _lib.check(_lib.lib().m25_getrf(_lib.P(F), ctypes.c_long(n), n, _lib.P(ipiv), 0, 0, _lib.P(work),
                                    ctypes.c_size_t(nb), _lib.stream_ptr()))
    del work
    for _ in range(2):                                               # twice: the flags' epochs
        X = R.clone()
        _lib.check(_lib.lib().m25_getrs(_lib.P(F), ctypes.c_long(n), n, _lib.P(ipiv), 0, _lib.P(X), nrhs,
                                        _lib.stream_ptr()))
        _lib.sync_check()
        err = (X - x).abs().max().item() / x.abs().max().item()
        assert err < 1e-11, err


@pytest.mark.parametrize('k', [1, 3, 8])
def test_gmres_batched_matches_a_direct_solve(small, k):
    """The refinement's GMRES (device Arnoldi steps, host least squares) on a dense system with a nearby
    preconditioner: every column converges to the direct solution; columns stop on their own at the tolerance."""
    geo, ds, od = small
    n = 400
    rng = np.random.default_rng(3 + k)
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 2 * np.sqrt(n) * np.eye(n)
    Pinv = np.linalg.inv(A + 3e-4 * np.abs(A).max() * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))))
    B = rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k))
    B[:, 0] *= 1e3                                         # columns of very different sizes
    Ad, Pd, Bd = (torch.from_numpy(x).to('cuda') for x in (A, Pinv, B))
    Y, it = ds.gmres_batched(lambda V: Ad @ V, Bd, lambda R: Pd @ R, rtol=1e-12, restart=30)
    X = np.linalg.solve(A, B)
    Yh = Y.cpu().numpy()
    assert (np.abs(Yh - X).max(0) <= 1e-9 * np.abs(X).max(0)).all(), it
    assert max(it) <= 20 and min(it) >= 1
    # a preconditioner that does not help within the stall rule's window ends the iteration early
    Y2, it2 = ds.gmres_batched(lambda V: Ad @ V, Bd, lambda R: 0 * R + R, rtol=1e-12, restart=30, stall=(4, 1e-9))
    assert max(it2) == 4
