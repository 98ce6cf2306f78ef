"""Wave ports through the whole GPU path: a microstrip between two wave ports (LinePort), its S-parameters
from Simulation.sparams (the device solve, then the feed fits and the balance) against the reference's own
Simulation.sparams on the same mesh (tests/golden/ports_golden.npz); solve_band renormalised to other reference
impedances against the reference's renorm of the same S; and line_char_xs on a microstrip against the
closed-form microstrip estimates (Hammerstad-Jensen; loose: the MoM line is not the formula's)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope='module')
def gold():
    return dict(np.load(os.path.join(HERE, 'golden', 'ports_golden.npz')))


@pytest.fixture(scope='module')
def wave_sim():
    from test_ports import _wave_board
    from mom25d_b200.sim import Simulation
    return Simulation.from_board(_wave_board(), precision='double')


def test_wave_port_sparams_match_the_reference(gold, wave_sim):
    for i, f in enumerate(gold['wave_f']):
        S = wave_sim.sparams(f)
        assert np.abs(S - gold['wave_S'][i]).max() <= 1e-8, f
        assert np.abs(wave_sim.last['gamma'] - gold['wave_gamma'][i]).max() <= 1e-6 * np.abs(gold['wave_gamma'][i]).max()
    wave_sim.precision = 'mixed'
    try:
        assert np.abs(wave_sim.sparams(gold['wave_f'][1]) - gold['wave_S'][1]).max() <= 1e-5
    finally:
        wave_sim.precision = 'double'


def test_solve_band_renormalises(gold, wave_sim):
    from mom25d_b200.run import renorm, solve_band
    f, S, info = solve_band(wave_sim, gold['wave_f'][0], gold['wave_f'][-1], zref=75.0, linear=2, log=lambda *a: None)
    assert np.allclose(f, [gold['wave_f'][0], gold['wave_f'][-1]])
    for j, i in ((0, 0), (1, 2)):
        assert np.abs(S[j] - renorm(gold['wave_S'][i], [50.0, 50.0], 75.0)).max() <= 1e-8
    assert info['zref'] == [75.0, 75.0] and info['solves'] == 2


def test_line_char_xs_microstrip_is_physical():
    from mom25d_b200.board import Layer, LayerStack, C0
    from mom25d_b200.ports import line_char_xs
    h, er, w = 0.8e-3, 4.4, 1.5e-3
    st = LayerStack([Layer(h, er, 0.0)])
    f = np.array([3e9, 6e9])                              # (the cuts span enough phase for the fit: FIT_SPAN)
    gam, zc = line_char_xs(st, 1, w, f, dmax=0.4e-3, length=24e-3)
    u = w / h                                             # Hammerstad-Jensen, zero thickness
    eeff = (er + 1) / 2 + (er - 1) / 2 * (1 + 10 / u) ** -0.555
    fu = 6 + (2 * np.pi - 6) * np.exp(-(30.666 / u) ** 0.7528)
    z0 = 60 / np.sqrt(eeff) * np.log(fu / u + np.sqrt(1 + (2 / u) ** 2))
    beta = 2 * np.pi * f / C0 * np.sqrt(eeff)
    assert np.all(np.abs(gam.imag / beta - 1) < 0.05), gam.imag / beta
    assert np.all(np.abs(zc.real / z0 - 1) < 0.15), (zc, z0)
    assert np.all(gam.real >= 0)
