"""Wave ports and S-parameter post-processing on the CPU, against fixtures the reference's own code wrote
(tests/golden/ports_golden.npz, made by tests/golden/make_ports.py): the feed's gamma and waves fitted on sample
cuts (base.py:161-172), the reciprocity balance (sim.py:1121-1143), renormalisation to other reference impedances
(run.py:14-23), and, for a microstrip between two wave ports, the gap and cut edges the mesh gives each port and
the S-matrix computed from the reference's own currents (sim.py:1045-1092)."""
import os

import numpy as np
import pytest

from mom25d_b200 import board as B
from mom25d_b200.geometry import Geometry
from mom25d_b200.ports import balance, fit_gamma, fit_waves
from mom25d_b200.run import renorm

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope='module')
def gold():
    return dict(np.load(os.path.join(HERE, 'golden', 'ports_golden.npz')))


def _wave_board():
    import importlib.util
    spec = importlib.util.spec_from_file_location('mp', os.path.join(HERE, 'golden', 'make_ports.py'))
    mp = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mp)
    return mp.wave_board(B)


def test_wave_fits_match_reference(gold):
    for case in range(3):
        Ik, s, step = gold[f'fit{case}_I'], gold[f'fit{case}_s'], float(gold[f'fit{case}_step'])
        g = fit_gamma(Ik, step)
        assert abs(g - complex(gold[f'fit{case}_gamma'])) <= 1e-12 * abs(g), case
        a, b = fit_waves(Ik, s - 2e-3, g)
        assert np.abs(a - gold[f'fit{case}_a']).max() <= 1e-10 * np.abs(a).max(), case
        assert np.abs(b - gold[f'fit{case}_b']).max() <= 1e-10 * np.abs(a).max(), case


def test_balance_matches_reference(gold):
    for case in range(3):
        exact = gold[f'bal{case}_exact']
        Sb, sc = balance(gold[f'bal{case}_S'], exact if exact.any() else None)
        assert np.abs(Sb - gold[f'bal{case}_Sb']).max() <= 1e-13, case
        assert np.abs(sc - gold[f'bal{case}_scale']).max() <= 1e-13, case
        assert np.abs(Sb - Sb.T).max() <= 1e-15


def test_renorm_matches_reference(gold):
    for case in range(3):
        out = renorm(gold[f'ren{case}_S'], gold[f'ren{case}_zc'], gold[f'ren{case}_zref'])
        assert np.abs(out - gold[f'ren{case}_out']).max() <= 1e-13, case
    S = gold['ren0_S']
    assert renorm(S, [50.0, 50.0], 50.0) is S                  # same impedances: unchanged


def test_wave_port_edges_and_s_from_the_reference_currents(gold):
    bd = _wave_board()
    assert np.array_equal(bd.nodes, gold['wave_nodes']) and np.array_equal(bd.tris, gold['wave_tris'])
    geo = Geometry(bd)
    assert np.allclose(np.array(geo.samples), gold['wave_samples'], rtol=0, atol=1e-15)
    for j in range(2):
        assert np.array_equal(geo.gaps[j][0], gold[f'wave_gap{j}'])
        for k, (idx, sig) in enumerate(geo.cuts[j]):
            assert np.array_equal(idx, gold[f'wave_cut{j}_{k}']) and np.array_equal(sig, gold[f'wave_cutsig{j}_{k}'])
    for i, f in enumerate(gold['wave_f']):
        info = {}
        S = geo.sparams_from_currents(gold['wave_I'][i], f, info)
        assert np.abs(S - gold['wave_S'][i]).max() <= 1e-12, f
        assert np.abs(info['gamma'] - gold['wave_gamma'][i]).max() <= 1e-10 * np.abs(gold['wave_gamma'][i]).max()


def test_line_port_sample_positions():
    p = B.LinePort(1, (0, 0), (0, 1), 1e-3, 3e-3, step=0.5e-3)
    assert np.allclose(p.sample_positions(0.3e-3), [1e-3, 1.5e-3, 2e-3, 2.5e-3, 3e-3])
    p = B.LinePort(1, (0, 0), (1, 0), 1e-3, 2e-3)                      # defaults: step dmax, s0 2 step, s1 ref
    assert np.allclose(p.sample_positions(0.4e-3), [0.8e-3, 1.2e-3, 1.6e-3, 2.0e-3])
    lines = B.port_lines([p, B.GapPort(2, (1e-3, 5e-3), (0, -1), 1e-3)], [], 0.4e-3)
    assert np.allclose(sorted(lines[1][0]), [0.0, 0.8e-3, 1.2e-3, 1.6e-3, 2.0e-3]) and lines[1][1] == []
    assert lines[2] == ([], [5e-3])
