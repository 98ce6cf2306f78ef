"""The oracle (a CPU restatement of the reference's hot path) pinned against the reference itself: its compiled
core built from its sources (oracle/_ref) and golden fixtures its own Python code wrote (tests/golden)."""
import numpy as np
import pytest

import oracle
from oracle import green, solve
from mom25d_b200 import board as B, geometry as G
from conftest import ref_core


def small_board():
    import importlib.util, os
    spec = importlib.util.spec_from_file_location('mg', os.path.join(os.path.dirname(__file__), 'golden',
                                                                     'make_golden.py'))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg.small_board(B)


def test_tensor_mesh_and_rwg_match_the_reference(golden):
    nd, tr = B.tensor_mesh([tuple(r) for r in golden['mesh_rects']], 0.4e-3, 6, 1.01 * max(1.1e-3, 0.6e-3),
                           [3.0e-3], [0.0], grade=1.0)
    assert np.array_equal(nd, golden['mesh_nodes']) and np.array_equal(tr, golden['mesh_tris'])
    r = B.RWG(nd, tr)
    for k in ('tp', 'tm', 'vp', 'vm', 'l', 'nrm'):
        assert np.array_equal(getattr(r, k), golden['rwg_' + k]), k


def test_board_packing_and_near_pairs_match_the_reference(golden):
    bd = small_board()
    assert np.array_equal(bd.nodes, golden['board_nodes']) and np.array_equal(bd.tris, golden['board_tris'])
    geo = G.Geometry(bd)
    for k in ('ep', 'em', 'lt', 'te', 'ta', 'tv', 'ap', 'am', 'vp', 'vm'):
        assert np.array_equal(geo.g[k], golden['board_g_' + k]), k
    P, Q = oracle.near_pairs(geo.g['cent'], geo.tri_size, geo.tri_z, geo.near_fac)
    assert np.array_equal(P, golden['board_nP']) and np.array_equal(Q, golden['board_nQ'])
    assert np.array_equal(geo.excitation(), golden['board_E'])


@pytest.mark.parametrize('name,o,s,xs,im', [('t11', 1, 1, False, True), ('t13', 1, 3, False, False),
                                            ('t23', 2, 3, True, False), ('t33', 3, 3, False, True)])
def test_green_tables_match_the_reference(golden, name, o, s, xs, im):
    st = B.LayerStack([B.Layer(0.2e-3, 3.5, 0.02), B.Layer(1.0e-3, 4.4, 0.02), B.Layer(0.2e-3, 3.5, 0.02)])
    gt = green.GreenTable(2.0e9, st, o, s, 12e-3, cross_sing=xs, image_sing=im)
    A, Q = golden[name + '_A'], golden[name + '_Q']
    assert np.abs(gt.A_rest[::16] - A).max() <= 1e-12 * np.abs(A).max()
    assert np.abs(gt.Q_rest[::16] - Q).max() <= 1e-12 * np.abs(Q).max()
    sc = np.array([gt.cA, gt.cq, gt.cAi, gt.cqi, gt.d, gt.dimg, gt.rho[1], gt.npts], complex)
    assert np.allclose(sc, golden[name + '_scal'], rtol=1e-12, atol=0)


def test_complex_bessel_matches_the_reference(golden):
    for n in range(3):
        assert np.array_equal(oracle.bessel_jn_complex(n, golden['jn_z']), golden['jn_%d' % n])


def test_oracle_kernels_match_the_reference_core_bit_for_bit():
    core = ref_core()
    if core is None:
        pytest.skip('oracle/_ref not built (oracle/build_ref.sh)')
    geo = G.Geometry(small_board())
    d = solve.Direct(geo)
    d.setup(3e9)
    Z1, Z2 = (np.zeros((geo.Ne, geo.Ne), complex) for _ in range(2))
    oracle.fill_far(Z1, geo.g, d.tb, d.w)
    core.fill_far(Z2, geo.g, d.tb, d.w)
    assert np.array_equal(Z1, Z2)
    q1 = oracle.near_into_dense(Z1, geo.g, d.tb, geo.q, d.nP32, d.nQ32, d.w)
    q2 = core.near_into_dense(Z2, geo.g, d.tb, geo.q, d.nP32, d.nQ32, d.w)
    assert np.abs(Z1 - Z2).max() <= 1e-15 * np.abs(Z2).max() and np.array_equal(q1, q2)   # (atomics' order)
    r1, c1, v1, _ = oracle.near_coo(geo.g, d.tb, geo.q, d.nP32, d.nQ32, d.w)
    r2, c2, v2, _ = core.near_coo(geo.g, d.tb, geo.q, d.nP32, d.nQ32, d.w)
    assert np.array_equal(r1, r2) and np.array_equal(c1[r1 >= 0], c2[r2 >= 0]) and np.array_equal(v1[r1 >= 0], v2[r2 >= 0])
    X = np.random.default_rng(0).normal(size=(geo.Ne, 3)) + 0j
    assert np.array_equal(oracle.matvec_far_multi(X, geo.g, d.tb, d.w), core.matvec_far_multi(X, geo.g, d.tb, d.w))
    F = np.asarray(geo.F, np.int32)
    assert np.array_equal(oracle.fan_q(geo.g, d.tb, F), core.fan_q(geo.g, d.tb, F))
    rows, cols = np.arange(0, geo.Ne, 3, dtype=np.int32), np.arange(0, geo.Ne, 5, dtype=np.int32)
    assert np.array_equal(oracle.far_block(rows, cols, geo.g, d.tb, d.w), core.far_block(rows, cols, geo.g, d.tb, d.w))
    rng = np.random.default_rng(1)
    Z = rng.normal(size=(40, 40)) + 1j * rng.normal(size=(40, 40))
    dd = rng.uniform(0.5, 2, 40)
    Za, Zb = Z.copy(), Z.copy()
    assert np.array_equal(oracle.scale_c64(Za, dd), core.scale_c64(Zb, dd)) and np.array_equal(Za, Zb)
    kr = np.linspace(1, 2e4, 500)
    W = rng.normal(size=(2, 500)) + 1j * rng.normal(size=(2, 500))
    rho = np.linspace(0, 5e-3, 33)
    assert np.array_equal(oracle.hankel_real(rho, kr, W), core.hankel_real(rho, kr, W))
    t = d.tb['A'][0]
    px, py, ww = geo.P6[:, :, 0], geo.P6[:, :, 1], geo.W6
    assert np.array_equal(oracle.radial_table_sum(px, py, ww, geo.ch_x, geo.ch_y, t, d.tb['dr'][0]),
                          core.radial_table_sum(px, py, ww, geo.ch_x, geo.ch_y, t, d.tb['dr'][0]))


def test_oracle_impedance_and_s_match_the_reference(golden):
    geo = G.Geometry(small_board())
    d = solve.Direct(geo)
    f = float(golden['board_f'][0])
    Z = d.impedance(f)
    Zr = golden['board_Z']
    assert np.linalg.norm(Z - Zr) <= 1e-12 * np.linalg.norm(Zr)
    S, X, _ = d.sparams(f)
    assert np.abs(S - golden['board_S_double']).max() < 1e-10
    assert np.abs(X - golden['board_I_double']).max() <= 1e-9 * np.abs(golden['board_I_double']).max()
    Sm, _, info = d.sparams(f, 'mixed')
    assert np.abs(Sm - golden['board_S_mixed']).max() < 1e-5 and max(info['iters']) <= 30


def test_oracle_gmres_matches_the_reference(golden):
    rng = np.random.default_rng(1)
    n = 200
    ev = (1 + rng.random(n)) * np.exp(1j * rng.uniform(-1.2, 1.2, n))
    Qm = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))[0]
    A = Qm @ np.diag(ev) @ Qm.conj().T + 0.2 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    Bm = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
    assert np.array_equal(Bm, golden['gmres_B'])
    X, it = solve.gmres_batched(lambda V: A @ V, Bm, rtol=1e-10, restart=60, maxiter=5)
    assert it == golden['gmres_it'].tolist()
    assert np.abs(X - golden['gmres_X']).max() <= 1e-12 * np.abs(X).max()
