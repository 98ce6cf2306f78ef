"""solve_band's adaptive sweep on the GPU (run.py:41-84 with afs.adaptive_sweep): on the golden board (two
interfaces, a via, two via ports) over 1-6 GHz, the S it returns at its solved frequencies equals a direct
solve there, and its model stays within afs_tol of direct solves spread over the whole output grid."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')


def test_adaptive_solve_band_matches_direct_solves():
    from test_gpu_parity import _small_board
    from mom25d_b200.run import solve_band
    from mom25d_b200.sim import Simulation
    sim = Simulation.from_board(_small_board(), precision='double')
    tol = 2e-3
    f, S, info = solve_band(sim, 1e9, 6e9, points=201, afs_tol=tol, log=None)
    assert info['afs'] and info['afs'][-1]['converged'] and info['solves'] < 40
    for fs in info['solved']:
        i = int(np.argmin(np.abs(f - fs)))
        if abs(f[i] - fs) <= 1e-9 * fs:
            assert np.abs(S[i] - sim.sparams(fs)).max() <= 1e-10
    check = range(0, len(f), 10)
    err = max(float(np.abs(S[i] - sim.sparams(f[i])).max()) for i in check)
    print(f"adaptive sweep: {info['solves']} solves, largest model error over {len(check)} checks {err:.1e}")
    assert err <= tol
