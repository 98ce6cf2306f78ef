"""The extra blocks of Z (mom25d_b200.extras; the reference's fast.py:628-641) on the CPU: the RWG Gram matrix of
the golden mesh, conductor surface impedances (plain, rough, with a finish) and R-L-C impedances against the
reference's own values (tests/golden/extras_golden.npz, made by tests/golden/make_extras.py), and the assembled
pattern for a meshed board with a lumped element: S = Zs Gram + Z(f) u u^T on the cut line's edges."""
import os

import numpy as np
import pytest

from mom25d_b200 import board as B
from mom25d_b200.extras import ExtraBlocks, Metal, SeriesLumped, gram_matrix, rlc

HERE = os.path.dirname(os.path.abspath(__file__))
METALS = [dict(), dict(sigma=5.8e7, t=18e-6, rough=1.2e-6),
          dict(sigma=5.8e7, t=35e-6, rough=0.5e-6, finish=[(1.45e7, 5e-6), (4.1e7, 0.1e-6)], on={3: 0.6})]
RLC = [dict(R=10.0, L=2e-9, C=1e-12), dict(R=50.0, L=1e-9, C=2e-12, parallel=True), dict(R=0.0, L=3e-9)]


@pytest.fixture(scope='module')
def gold():
    return np.load(os.path.join(HERE, 'golden', 'extras_golden.npz'))


def test_gram_matrix_matches_reference(gold):
    g = np.load(os.path.join(HERE, 'golden', 'reference_golden.npz'))
    rwg = B.RWG(g['mesh_nodes'], g['mesh_tris'])
    assert rwg.Ne == int(gold['gram_ne'])
    r, c, v = gram_matrix(rwg, B.quad_pts(rwg, B.BAR3), B.W3)
    G = np.zeros((rwg.Ne, rwg.Ne))
    G[r, c] = v
    ref = np.zeros_like(G)
    ref[gold['gram_rows'], gold['gram_cols']] = gold['gram_vals']
    big = 1e-12 * np.abs(ref).max()                    # (entries that vanish analytically differ in rounding noise)
    assert np.array_equal(np.abs(G) > big, np.abs(ref) > big)
    assert np.abs(G - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.abs(G - G.T).max() <= 1e-15 * np.abs(G).max()


def test_surface_impedance_and_rlc_match_reference(gold):
    for i, kw in enumerate(METALS):
        m = Metal(**kw)
        for k, key in ((None, f'zs_{i}'), (3, f'zs_{i}_k3')):
            z = np.array([m.zs(f, k) for f in gold['freqs']])
            assert np.abs(z - gold[key]).max() <= 1e-13 * np.abs(gold[key]).max(), key
    for i, kw in enumerate(RLC):
        z = np.array([rlc(**kw)(f) for f in gold['freqs']])
        assert np.abs(z - gold[f'rlc_{i}']).max() <= 1e-13 * np.abs(gold[f'rlc_{i}']).max()


def test_extra_blocks_pattern_and_values():
    from mom25d_b200.geometry import Geometry
    st = B.LayerStack([B.Layer(0.8e-3, 4.4, 0.02)])
    rects = {1: [(-6e-3, -0.75e-3, 6e-3, 0.75e-3)]}
    el = SeriesLumped(1, (0.0, 0.0), (1.0, 0.0), 1.5e-3, rlc(R=25.0, L=1e-9), 'R1')
    nodes, tris, tl = B.mesh_layers(st, rects, 0.5e-3, lines={1: ([0.0], [])})
    bd = B.Board(st, nodes, tris, tl, [], [B.GapPort(1, (-5e-3, 0.0), (1.0, 0.0), 1.5e-3)], 0.5e-3, 5.0, 'strip',
                 rects)
    geo = Geometry(bd)
    metal = Metal(sigma=5.8e7, t=35e-6, rough=1e-6, finish=[(4.1e7, 0.1e-6)], on={1: 0.5})
    ex = ExtraBlocks(geo, [el], metal)
    f = 2.5e9
    S = ex.dense(f)
    idx, sig = geo.gap_edges(el.lp)
    assert len(idx) >= 2
    r, c, v = gram_matrix(geo.rwg, B.quad_pts(geo.rwg, B.BAR3), B.W3)
    zs = metal.zs_edges(f, geo.edge_layer)
    ref = np.zeros((geo.N, geo.N), complex)
    ref[r, c] = (zs[r] if np.ndim(zs) else zs) * v
    u = sig * geo.rwg.l[idx]
    ref[np.ix_(idx, idx)] += el.Z(f) * np.outer(u, u)
    assert np.abs(S - ref).max() <= 1e-14 * np.abs(ref).max()
    assert len(np.unique(ex.ri.astype(np.int64) * geo.N + ex.ci)) == ex.nnz       # distinct entries
    assert ExtraBlocks(geo).nnz == 0
