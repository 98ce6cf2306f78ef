"""The extra blocks of Z on the GPU (fast.py:628-641): a strip with a series R-L element across its middle and
conductor loss with a partial surface finish. The filled Z minus the same fill without them is the host's S
(complex128 to its rounding; complex64 to single precision), and the S-parameters of the double and the mixed
(hybrid) solves agree, so the factor and the refinement's operator both carry the additions."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')


@pytest.fixture(scope='module')
def strip():
    from mom25d_b200 import board as B
    from mom25d_b200.extras import Metal, SeriesLumped, rlc
    st = B.LayerStack([B.Layer(0.8e-3, 4.4, 0.02)])
    rects = {1: [(-6e-3, -0.75e-3, 6e-3, 0.75e-3)]}
    el = SeriesLumped(1, (0.0, 0.0), (1.0, 0.0), 1.5e-3, rlc(R=25.0, L=1e-9), 'R1')
    nodes, tris, tl = B.mesh_layers(st, rects, 0.4e-3, lines={1: ([-5e-3, 0.0, 5e-3], [])})
    ports = [B.GapPort(1, (-5e-3, 0.0), (1.0, 0.0), 1.5e-3, 50.0, 'P1'),
             B.GapPort(1, (5e-3, 0.0), (1.0, 0.0), 1.5e-3, 50.0, 'P2')]
    bd = B.Board(st, nodes, tris, tl, [], ports, 0.4e-3, 5.0, 'strip', rects)
    metal = Metal(sigma=5.8e7, t=35e-6, rough=1e-6, finish=[(4.1e7, 0.1e-6)], on={1: 0.5})
    return bd, el, metal


def test_z_carries_the_extra_blocks(strip):
    from mom25d_b200.sim import Simulation
    bd, el, metal = strip
    f = 3e9
    plain = Simulation.from_board(bd, precision='double')
    extra = Simulation.from_board(bd, precision='double', lumped=[el], metal=metal)
    S = extra.fast.extras.dense(f)
    for prec, tol in (('double', 1e-15), ('mixed', 2 ** -22)):
        Zo = plain.fast.impedance(f, prec).clone().cpu().numpy().astype(complex)
        Zw = extra.fast.impedance(f, prec).clone().cpu().numpy().astype(complex)
        assert np.abs(Zw - Zo - S).max() <= tol * np.abs(Zo).max() + 1e-12 * np.abs(S).max(), prec
    assert np.abs(S).max() > 0


def test_double_and_mixed_agree_with_the_extra_blocks(strip):
    from mom25d_b200.sim import Simulation
    bd, el, metal = strip
    d = Simulation.from_board(bd, precision='double', lumped=[el], metal=metal)
    m = Simulation.from_board(bd, precision='mixed', lumped=[el], metal=metal)
    for f in (1e9, 4e9):
        Sd, Sm = d.sparams(f), m.sparams(f)
        assert np.abs(Sd - Sm).max() <= 1e-5
    plain = Simulation.from_board(bd, precision='double')
    assert np.abs(plain.sparams(4e9) - Sd).max() > 1e-3      # the 25 ohm element is seen in S
