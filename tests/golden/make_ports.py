"""
Generates tests/golden/ports_golden.npz from the reference's own code (lowprocess/mom25d, read-only checkout): its
wave fits on a feed (base.py:161-172 fit_gamma, fit_waves) on synthetic two-wave currents, its reciprocity balance
(sim.py:1121-1143) on random S-matrices, and the S-parameters of a microstrip with a wave port (LinePort) at each
end, solved by its own Simulation.sparams (direct solver, double precision) on the mesh this package's tensor
mesher makes with the ports' sample lines (bit-exact with the reference's mesher on rectangles).

    python tests/golden/make_ports.py [/path/to/reference]

Run in this container only; the reference's modules import with shapely and emsdev stubbed as in make_golden.py,
and its Simulation is made with __new__ from the same mesh (its constructor needs shapely).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = sys.argv[1] if len(sys.argv) > 1 else '/root/reference'
sys.path.insert(0, HERE)
from make_golden import _stubs                                      # noqa: E402

FREQS = np.array([1.5e9, 4.0e9, 7.5e9])


def wave_board(B):
    """A 12.8 mm x 1.5 mm strip on one layer (h = 0.8 mm, er = 4.4, tan d = 0.02); a wave port 0.4 mm inside each
    end, feeding inward, reference plane 2.4 mm in, sample cuts every 0.4 mm (the default step, dmax)."""
    st = B.LayerStack([B.Layer(0.8e-3, 4.4, 0.02)])
    rects = {1: [(-6.4e-3, -0.75e-3, 6.4e-3, 0.75e-3)]}
    dmax = 0.4e-3
    ports = [B.LinePort(1, (-6.0e-3, 0.0), (1.0, 0.0), 1.5e-3, 2.4e-3, zc=50.0, name='P1'),
             B.LinePort(1, (6.0e-3, 0.0), (-1.0, 0.0), 1.5e-3, 2.4e-3, zc=50.0, name='P2')]
    nodes, tris, tl = B.mesh_layers(st, rects, dmax, lines=B.port_lines(ports, [], dmax))
    return B.Board(st, nodes, tris, tl, [], ports, dmax, 5.0, 'wave_board', rects)


def main():
    _stubs()
    sys.path.insert(0, os.path.join(REF, 'src'))
    sys.path.insert(0, os.path.join(REPO, 'oracle', '_ref'))
    sys.path.insert(0, REPO)
    import _core
    sys.modules['mom25d._core'] = _core
    import mom25d
    mom25d._core = _core
    from mom25d import fast, sim as rsim, multilayer as rml, base as rbase, geo as rgeo
    from mom25d_b200 import board as B, geometry as G

    out = {}
    rng = np.random.default_rng(7)
    # 1. wave fits: I(s) = a e^{-g s} + b e^{g s} (+ a little noise), several columns
    for case, (g, step, n, cols) in enumerate([(0.05 + 80j, 0.4e-3, 6, 2), (2.0 + 150j, 0.25e-3, 9, 3),
                                               (0.01 + 20j, 1.0e-3, 5, 1)]):
        s = step * np.arange(n) + 0.8e-3
        a = rng.standard_normal(cols) + 1j * rng.standard_normal(cols)
        b = 0.3 * (rng.standard_normal(cols) + 1j * rng.standard_normal(cols))
        Ik = np.exp(-g * s)[:, None] * a + np.exp(g * s)[:, None] * b
        Ik = Ik + 1e-4 * (rng.standard_normal(Ik.shape) + 1j * rng.standard_normal(Ik.shape))
        gf = rbase.fit_gamma(Ik, step)
        A_, B_ = rbase.fit_waves(Ik, s - 2e-3, gf)
        out.update({f'fit{case}_I': Ik, f'fit{case}_s': s, f'fit{case}_step': np.array(step),
                    f'fit{case}_gamma': np.array(gf), f'fit{case}_a': A_, f'fit{case}_b': B_})
    # 2. balance on random S with a diagonal scale error, with and without exact (lumped) ports
    for case, n in enumerate([2, 4, 5]):
        S0 = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        S0 = 0.3 * (S0 + S0.T)
        d = np.exp(0.2 * rng.standard_normal(n))
        S = S0 * (d[:, None] / d[None, :])
        exact = np.arange(n) % 3 == 2
        Sb, sc = rsim.balance(S, exact if exact.any() else None)
        out.update({f'bal{case}_S': S, f'bal{case}_exact': exact, f'bal{case}_Sb': Sb, f'bal{case}_scale': sc})
    # 3. renormalisation to other reference impedances (run.py:14-23)
    from mom25d import run as rrun
    for case, (zc, zref) in enumerate([([50.0, 50.0], [75.0, 75.0]), ([50.0, 75.0, 30.0], 50.0),
                                       ([42.0, 61.0], [50.0, 100.0])]):
        n = len(zc)
        S0 = 0.4 * (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
        S0 = 0.5 * (S0 + S0.T)
        out.update({f'ren{case}_S': S0, f'ren{case}_zc': np.array(zc), f'ren{case}_zref': np.broadcast_to(zref, n),
                    f'ren{case}_out': rrun.renorm(S0, zc, zref)})
    # 4. a microstrip between two wave ports, the reference's own sparams
    bd = wave_board(B)
    geo = G.Geometry(bd)
    s = rsim.Simulation.__new__(rsim.Simulation)
    stack = rml.LayerStack([rml.Layer(l.h, l.er, l.tand) for l in bd.stack.layers])
    ports = [rgeo.LinePort(p.layer, tuple(p.c), tuple(p.d), p.w, p.ref, zc=p.zc, name=p.name) for p in bd.ports]
    samples = []
    for p in ports:                                          # sim.py:426-431 with the defaults
        step = p.step or bd.dmax
        s0, s1 = (p.s0 if p.s0 is not None else 2 * step), (p.s1 if p.s1 is not None else p.ref)
        samples.append(s1 - step * np.arange(int(np.floor((s1 - s0) / step + 1e-9)) + 1)[::-1])
    s.__dict__.update(st=stack, rwg=rbase.RWG(bd.nodes, bd.tris), tri_layer=bd.tri_layer, layers=geo.layers,
                      Ne=geo.Ne, Nv=0, near_fac=5.0, dmax=bd.dmax, P3=geo.P3, W3=geo.W3, P6=geo.P6, W6=geo.W6,
                      tri_size=geo.tri_size, log=rml.RunLog(False), F=geo.F, dF=geo.dF, lumped=[], lumped_edges=[],
                      metal=None, qT=None, gpu='off', reuse='off', stream='off', loop_tree='off', frills=[], slots=[],
                      chains=[], vias=[], rho_max=geo.rho_max, tri_idx=geo.tri_idx, ports=ports, samples=samples,
                      tables={}, solver='direct', precision='double', _gram=None, _xcache={}, _slot_cache={},
                      edge_layer=geo.edge_layer, user_ports=ports)
    s._edge_sets()
    s.fast = fast.FastOperator(s)
    Ss, Is, gams = [], [], []
    for f in FREQS:
        Ss.append(s.sparams(f, keep=True))
        Is.append(s.last['I'])
        gams.append(s.last['gamma'])
    out.update(wave_f=FREQS, wave_S=np.array(Ss), wave_I=np.array(Is), wave_gamma=np.array(gams),
               wave_nodes=bd.nodes, wave_tris=bd.tris, wave_samples=np.array(samples))
    for j in range(len(ports)):
        out[f'wave_gap{j}'] = s.gap[j][0]
        for k, (idx, sig) in enumerate(s.cuts[j]):
            out[f'wave_cut{j}_{k}'] = idx
            out[f'wave_cutsig{j}_{k}'] = sig
    np.savez_compressed(os.path.join(HERE, 'ports_golden.npz'), **out)
    print('wrote ports_golden.npz: N =', geo.N, 'S(1.5 GHz) =', np.round(Ss[0], 4).tolist())


if __name__ == '__main__':
    main()
