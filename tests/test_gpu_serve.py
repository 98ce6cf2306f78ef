"""The serving loop on the GPU: requests for two resident boards run concurrently on several streams, and each
request's S is the same alone and in the mix (within 1e-7: the mix changes only the order of the near field's
atomic additions), and agrees with the FP64 solve to the mixed-precision bar."""
import importlib.util
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')


def _boards():
    from mom25d_b200 import board as B
    spec = importlib.util.spec_from_file_location('mg', os.path.join(os.path.dirname(__file__), 'golden',
                                                                     'make_golden.py'))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return {'vias': mg.small_board(B), 'strip': B.microstrip_board(dmax=1.0e-3, length=20e-3)}


def test_each_result_is_the_same_alone_and_in_the_mix():
    from mom25d_b200.serve import Request, Server
    from mom25d_b200.geometry import Geometry
    from mom25d_b200.operator import DirectSolver
    boards = _boards()
    plan = [('vias', 2.0e9), ('strip', 1.5e9), ('vias', 3.0e9), ('strip', 4.0e9), ('vias', 5.0e9), ('strip', 2.5e9)]
    alone = {}
    srv1 = Server(boards, slots=1)
    for i, (k, f) in enumerate(plan):
        r = srv1.run([Request(i, k, f)])[0]
        assert r.error is None, r.error
        alone[i] = r.S
    mix = Server(boards, slots=3).run([Request(i, k, f, 0.0) for i, (k, f) in enumerate(plan)])
    assert len({r.slot for r in mix}) > 1                          # they did share the device
    for r in mix:
        assert r.error is None, r.error
        assert np.abs(r.S - alone[r.rid]).max() <= 1e-7
    for i, (k, f) in enumerate(plan[:2]):                          # against the FP64 drop-in path
        geo = Geometry(boards[k])
        S64 = geo.sparams_from_currents(DirectSolver(geo).solve_direct(f, geo.excitation(), precision='double')
                                        .cpu().numpy())
        assert np.abs(alone[i] - S64).max() <= 1e-5
