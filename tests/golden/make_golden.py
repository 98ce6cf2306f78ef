"""
Generates the golden fixtures in tests/golden/ by importing the reference (lowprocess/mom25d) from its read-only
checkout and running its own code: its mesher, RWG basis, Green tables, compiled core (built from its sources by
oracle/build_ref.sh into oracle/_ref/), via blocks, batched GMRES and its direct solver (double and mixed).

    python tests/golden/make_golden.py [/path/to/reference]

The reference's Simulation constructor needs shapely and emsdev (absent here); the few attributes its solver reads
are set on an instance made with __new__ instead, from the same mesh. shapely and emsdev are stubbed only so its
modules import. Run in this container only (the reference does not exist on the GPU box); the fixtures it writes
are small .npz files committed with it.
"""
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = sys.argv[1] if len(sys.argv) > 1 else '/root/reference'


def _stubs():
    sh = types.ModuleType('shapely')
    for sub in ('geometry', 'ops', 'affinity'):
        m = types.ModuleType('shapely.' + sub)
        setattr(sh, sub, m)
        sys.modules['shapely.' + sub] = m
    for n in ('LineString', 'Point', 'Polygon', 'box', 'shape', 'MultiPolygon'):
        setattr(sys.modules['shapely.geometry'], n, object)
    sys.modules['shapely.ops'].unary_union = None
    sys.modules['shapely'] = sh
    em = types.ModuleType('emsdev')
    mem = types.ModuleType('emsdev.memory')
    mem.available = lambda: 64e9
    gpu = types.ModuleType('emsdev.gpu')
    gpu.Unavailable = RuntimeError
    em.memory, em.gpu = mem, gpu
    sys.modules.update({'emsdev': em, 'emsdev.memory': mem, 'emsdev.gpu': gpu})


def main():
    _stubs()
    sys.path.insert(0, os.path.join(REF, 'src'))
    sys.path.insert(0, os.path.join(REPO, 'oracle', '_ref'))
    sys.path.insert(0, REPO)
    import _core
    sys.modules['mom25d._core'] = _core
    import mom25d
    mom25d._core = _core
    from mom25d import fast, sim as rsim, multilayer as rml, base as rbase, via as rvia
    from mom25d_b200 import board as B, geometry as G

    out = {}
    # 1. the tensor mesher and the RWG basis (multilayer.py:338, base.py:16)
    rects = [(-4e-3, -0.55e-3, 4e-3, 0.55e-3), (-0.55e-3, 0.55e-3, 0.55e-3, 3.2e-3)]
    nd, tr = rml.make_mesh_ml(rects, 0.4e-3, 6, 1.01 * max(1.1e-3, 0.6e-3), [3.0e-3], [0.0], grade=1.0)
    r = rbase.RWG(nd, tr)
    out.update(mesh_rects=np.array(rects), mesh_nodes=nd, mesh_tris=tr, rwg_tp=r.tp, rwg_tm=r.tm, rwg_vp=r.vp,
               rwg_vm=r.vm, rwg_l=r.l, rwg_nrm=r.nrm)

    # 2. Green tables of the 3-layer stack: same interface with image, cross plain, cross extracted
    st = rml.LayerStack([rml.Layer(0.2e-3, 3.5, 0.02), rml.Layer(1.0e-3, 4.4, 0.02), rml.Layer(0.2e-3, 3.5, 0.02)])
    f = 2.0e9
    for name, (o, s, xs, im) in dict(t11=(1, 1, False, True), t13=(1, 3, False, False), t23=(2, 3, True, False),
                                     t33=(3, 3, False, True)).items():
        gt = rml.GreenTableML(f, st, o, s, 12e-3, cross_sing=xs, image_sing=im)
        out[name + '_A'], out[name + '_Q'] = gt.A_rest[::16].copy(), gt.Q_rest[::16].copy()
        out[name + '_scal'] = np.array([gt.cA, gt.cq, gt.cAi, gt.cqi, gt.d, gt.dimg, gt.rho[1], gt.npts], complex)

    # 3. a small two-interface board with vias and via ports, solved by the reference's direct solver
    bd = small_board(B)
    geo = G.Geometry(bd)
    s = rsim.Simulation.__new__(rsim.Simulation)
    stack = rml.LayerStack([rml.Layer(l.h, l.er, l.tand) for l in bd.stack.layers])
    vias = [rsim.Via(v.x, v.y, v.k_bot, v.k_top, v.a, name=v.name) for v in bd.vias]
    chains = [(vias[bd.vias.index(v)], kb, kt) for v, kb, kt in geo.chains]
    ports = [rsim.ViaPort(vias[bd.vias.index(p.via)], p.zc, p.name) for p in bd.ports]
    s.__dict__.update(st=stack, rwg=rbase.RWG(bd.nodes, bd.tris), tri_layer=bd.tri_layer, layers=geo.layers,
                      Ne=geo.Ne, Nv=geo.Nv, near_fac=5.0, dmax=bd.dmax, P3=geo.P3, W3=geo.W3, P6=geo.P6, W6=geo.W6,
                      tri_size=geo.tri_size, log=rml.RunLog(False), F=geo.F, dF=geo.dF, lumped=[], lumped_edges=[],
                      metal=None, qT=None, gpu='off', reuse='off', stream='off', loop_tree='off', frills=[], slots=[],
                      chains=chains, vias=vias, rho_max=geo.rho_max, tri_idx=geo.tri_idx, ports=ports,
                      samples=[None] * len(ports), gap=[None] * len(ports), cuts=[None] * len(ports), tables={},
                      solver='direct', precision='double', _gram=None, _xcache={}, _slot_cache={},
                      edge_layer=geo.edge_layer, user_ports=ports)
    s.fast = fast.FastOperator(s)
    fo = s.fast
    out.update(board_nodes=bd.nodes, board_tris=bd.tris, board_tri_layer=bd.tri_layer, board_nP=fo.nP, board_nQ=fo.nQ)
    for k in ('ep', 'em', 'lt', 'te', 'ta', 'tv', 'ap', 'am', 'vp', 'vm'):
        out['board_g_' + k] = fo.g[k]
    fb = 3.0e9
    fo.setup(fb, mode='direct')
    N = geo.Ne + geo.Nv
    Z = np.zeros((N, N), complex)
    _core.fill_far(Z, fo.g, fo.tb, fo.w)
    fo._qcorr = _core.near_into_dense(Z, fo.g, fo.tb, fo.q, fo.nP32, fo.nQ32, fo.w)
    fo._vias(fb)
    Z[:geo.Ne, geo.Ne:], Z[geo.Ne:, :geo.Ne], Z[geo.Ne:, geo.Ne:] = fo.B, fo.B.T, fo.C
    out['board_Z'] = Z
    for k in ('A', 'Q'):
        out['board_tb_' + k] = fo.tb[k][:, ::16].copy()
    for k in ('cA', 'cq', 'cAi', 'cqi', 'dr', 'd', 'dimg', 'kind', 'tab'):
        out['board_tb_' + k] = fo.tb[k]
    out['board_E'] = s.excitation()
    s.precision = 'double'
    out['board_S_double'] = s.sparams(fb)
    out['board_I_double'] = s.fast.solve_direct(fb, s.excitation(), precision='double')
    s.precision = 'mixed'
    out['board_S_mixed'] = s.sparams(fb)
    out['board_f'] = np.array([fb])

    # 4. batched GMRES on the reference's own test system (test_solver.py:375-398)
    rng = np.random.default_rng(1)
    n = 200
    ev = (1 + rng.random(n)) * np.exp(1j * rng.uniform(-1.2, 1.2, n))
    Qm = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))[0]
    A = Qm @ np.diag(ev) @ Qm.conj().T + 0.2 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) / np.sqrt(n)
    Bm = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
    X, it = fast.gmres_batched(lambda V: A @ V, Bm, rtol=1e-10, restart=60, maxiter=5)
    out.update(gmres_B=Bm, gmres_X=X, gmres_it=np.array(it))   # A: regenerated from the seed by the test

    # 5. J_n of complex argument and the real-axis Hankel sum (via.py:56-101)
    z = (np.linspace(0.01, 30, 64) * np.exp(1j * np.linspace(0, 0.6, 64)))
    out.update(jn_z=z, jn_0=_core.bessel_jn_complex(0, z), jn_1=_core.bessel_jn_complex(1, z),
               jn_2=_core.bessel_jn_complex(2, z))
    np.savez_compressed(os.path.join(HERE, 'reference_golden.npz'), **out)
    print('wrote', os.path.join(HERE, 'reference_golden.npz'), 'N =', N)


def small_board(B):
    """A 4 mm strip on the top interface over a plane on interface 1 with a via between them at one end and two
    ground-referenced via ports: every table kind the configs use (same interface with image; cross plain)."""
    st = B.LayerStack([B.Layer(0.2e-3, 3.5, 0.02), B.Layer(1.0e-3, 4.4, 0.02), B.Layer(0.2e-3, 3.5, 0.02)])
    rects = {1: [(-1.0e-3, -1.5e-3, 3.0e-3, 1.5e-3)], 3: [(-2.4e-3, -0.4e-3, 2.4e-3, 0.4e-3)]}
    v = B.Via(2.0e-3, 0.0, 1, 3, 0.15e-3, 'V1')
    p1 = B.Via(-2.0e-3, 0.0, 0, 3, 0.15e-3, 'P1')
    p2 = B.Via(0.0, 1.0e-3, 0, 1, 0.15e-3, 'P2')
    vias = [p1, p2, v]
    nodes, tris, tl = B.mesh_layers(st, rects, 0.4e-3, ncross=3, vias=vias)
    return B.Board(st, nodes, tris, tl, vias, [B.ViaPort(p1, 50.0, 'P1'), B.ViaPort(p2, 50.0, 'P2')], 0.4e-3, 5.0,
                   'small', rects)


if __name__ == '__main__':
    main()
