"""
Generates tests/golden/extras_golden.npz from the reference's own code (lowprocess/mom25d, read-only checkout):
the RWG Gram matrix of the golden mesh (base.py:153-157), conductor surface impedances (sim.py:228-270: plain,
rough, and with a surface finish on one interface) and R-L-C element impedances (sim.py:48-56).

    python tests/golden/make_extras.py [/path/to/reference]

Run in this container only; the reference's modules import with shapely and emsdev stubbed as in make_golden.py.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else '/root/reference'
sys.path.insert(0, HERE)
from make_golden import _stubs                                      # noqa: E402

FREQS = np.array([1e8, 1e9, 3e9, 1e10])
METALS = [dict(), dict(sigma=5.8e7, t=18e-6, rough=1.2e-6),
          dict(sigma=5.8e7, t=35e-6, rough=0.5e-6, finish=[(1.45e7, 5e-6), (4.1e7, 0.1e-6)], on={3: 0.6})]
RLC = [dict(R=10.0, L=2e-9, C=1e-12), dict(R=50.0, L=1e-9, C=2e-12, parallel=True), dict(R=0.0, L=3e-9)]


def main():
    _stubs()
    sys.path.insert(0, os.path.join(REF, 'src'))
    from mom25d import base as rbase, sim as rsim
    g = np.load(os.path.join(HERE, 'reference_golden.npz'))
    rwg = rbase.RWG(g['mesh_nodes'], g['mesh_tris'])
    G = np.asarray(rbase.gram_matrix(rwg))
    r, c = np.nonzero(G)
    out = dict(gram_rows=r, gram_cols=c, gram_vals=G[r, c], gram_ne=np.array(rwg.Ne), freqs=FREQS)
    for i, kw in enumerate(METALS):
        m = rsim.Metal(**kw)
        out[f'zs_{i}'] = np.array([m.zs(f) for f in FREQS])
        out[f'zs_{i}_k3'] = np.array([m.zs(f, 3) for f in FREQS])
    for i, kw in enumerate(RLC):
        Z = rsim.rlc(**kw)
        out[f'rlc_{i}'] = np.array([Z(f) for f in FREQS])
    np.savez_compressed(os.path.join(HERE, 'extras_golden.npz'), **out)
    print({k: np.shape(v) for k, v in out.items()})


if __name__ == '__main__':
    main()
