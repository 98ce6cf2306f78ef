"""The FP64 drop-in against the reference's CPU path on the benchmark boards themselves, not only on the small
golden board: the 2-port microstrip through line (1 layer, dmax 0.3 mm), the stub notch filter (3 layers,
dmax 0.2 mm) and the seeded routed board (24 traces, 16 vias, 8 ports, N = 18,788).

The reference side is its compiled core (oracle/_ref, built from its sources; the oracle's C restatement of it,
pinned bit-exact in test_oracle.py, where that was not built) for the far fill and the near correction, the
oracle's restatement of its Green tables and via blocks, and LAPACK zgetrf / zgetrs of Z^T through SciPy, the
reference's own call (fast.py:318-358). The GPU side is the library through its C ABI.

Bars (the drop-in's): Z relative Frobenius difference <= 1e-10, max |dS| <= 1e-8; the mixed path's S within
1e-4 of the reference's double S."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')


def _reference_sweep(geo):
    from conftest import ref_core
    from oracle import solve as osolve
    import oracle
    core = ref_core()
    return osolve.KeptSweep(geo, core=core if core is not None else oracle)


def _boards():
    from mom25d_b200 import board as B
    return {'microstrip': lambda: B.microstrip_board(dmax=0.3e-3),
            'stub_filter': lambda: B.stub_filter_board(dmax=0.2e-3),
            'routed_board': lambda: B.routed_board(seed=1, ncross=4)}


CASES = [('microstrip', 1.0e9), ('microstrip', 3.5e9), ('microstrip', 6.0e9),
         ('stub_filter', 1.0e9), ('stub_filter', 6.0e9),
         ('routed_board', 0.5e9), ('routed_board', 10.0e9)]
_cache = {}


def _setup(name):
    if name not in _cache:
        from mom25d_b200.geometry import Geometry
        from mom25d_b200.sim import Simulation
        bd = _boards()[name]()
        sim = Simulation.from_board(bd, precision='double')
        _cache.clear()                                   # one board's buffers at a time
        _cache[name] = (sim, _reference_sweep(sim.geo))
    return _cache[name]


@pytest.mark.parametrize('name,f', CASES)
def test_fp64_drop_in_matches_the_reference_cpu_path(name, f):
    sim, ref = _setup(name)
    geo, ds = sim.geo, sim.fast
    Zg = ds.impedance(f, 'double')
    Zr = ref.impedance(f)
    Zr_dev = torch.from_numpy(Zr).to('cuda')
    z_rel = float(torch.linalg.norm(Zg - Zr_dev) / torch.linalg.norm(Zr_dev))
    del Zr_dev
    E = geo.excitation()
    Xr = ref.solve_z(f, Zr, E, precision='double')
    del Zr
    S_ref = geo.sparams_from_currents(Xr)
    S_gpu = geo.sparams_from_currents(ds.solve_direct(f, E, precision='double').cpu().numpy())
    dS = float(np.abs(S_gpu - S_ref).max())
    print(f"{name} N={geo.N} {f / 1e9:g} GHz: Z rel-Frobenius {z_rel:.2e}, max|dS| {dS:.2e}")
    assert z_rel <= 1e-10, z_rel
    assert dS <= 1e-8, dS
    if geo.N > 3500:                                     # the reference's mixed default above 3,500 unknowns
        ds.kept, ds.mixed_failed = [], 0.0
        S_mix = geo.sparams_from_currents(ds.solve_direct(f, E, precision='mixed').cpu().numpy())
        assert np.abs(S_mix - S_ref).max() <= 1e-4
