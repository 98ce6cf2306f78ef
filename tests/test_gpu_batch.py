"""The batched sweep on the GPU (mom25d_b200.batch.run): a coarse stub filter board at six frequencies on three
slots. Every batched result (a fresh complex64 LU each) agrees with the FP64 drop-in path to 1e-5, and the
sequential mixed sweep with kept-LU reuse (GMRES to a 1e-6 residual from a neighbouring frequency's factor) to
the metric's bar, |dS| <= 1e-4."""
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
