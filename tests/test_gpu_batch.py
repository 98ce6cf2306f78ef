"""The batched sweep on the GPU (mom25d_b200.batch.run): a coarse stub filter board at six frequencies on three
slots. The far part of every frequency's Z comes from one multi-frequency launch (m25_fill_far_multi), equal to
the per-frequency fills; every batched result (a fresh complex64 LU each) agrees with the FP64 drop-in path to
1e-5, and the sequential mixed sweep with kept-LU reuse (GMRES to a 1e-6 residual from a neighbouring frequency's
factor) to the metric's bar, |dS| <= 1e-4."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')


def test_batched_sweep_matches_fp64():
    from mom25d_b200.batch import run
    from mom25d_b200.board import stub_filter_board
    bd = stub_filter_board(dmax=0.6e-3)
    out = run(bd, np.linspace(1e9, 6e9, 6), slots=3)
    assert out['frequencies'] == 6 and out['fp64']['frequencies'] == 6
    assert out['max_dS_batched_vs_fp64'] <= 1e-5
    assert out['max_dS_sequential_mixed_vs_fp64'] <= 1e-4
    assert out['batched']['solves_per_s'] > 0 and out['fp64']['solves_per_s'] > 0


def test_multi_frequency_fill_equals_per_frequency_fills():
    import ctypes
    from mom25d_b200 import _lib
    from mom25d_b200.batch import fill_far_sweep
    from mom25d_b200.board import stub_filter_board
    from mom25d_b200.device import DeviceGeometry
    from mom25d_b200.geometry import Geometry
    geo = Geometry(stub_filter_board(dmax=0.6e-3))
    dg = DeviceGeometry(geo)
    freqs = [1.0e9, 2.7e9, 6.0e9]
    Zs, tabs = fill_far_sweep(geo, dg, freqs)
    Ne, N = geo.Ne, geo.N
    for f, Z, tb in zip(freqs, Zs, tabs):
        Z1 = torch.zeros((N, N), dtype=torch.complex128, device='cuda')
        _lib.check(_lib.lib().m25_fill_far(_lib.P(Z1), ctypes.c_long(N), 0, ctypes.byref(dg.mesh),
                                           ctypes.byref(tb.tables), None, ctypes.c_double(2 * np.pi * f),
                                           _lib.stream_ptr()), 'm25_fill_far')
        torch.cuda.synchronize()
        a, b = Z[:Ne, :Ne], Z1[:Ne, :Ne]
        assert float((a - b).abs().max()) <= 1e-12 * float(b.abs().max()), f
