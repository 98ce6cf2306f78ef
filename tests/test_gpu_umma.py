"""The complex64 LU's trailing update on the tensor cores (tcgen05, 3xTF32) against a NumPy double product."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')


@pytest.mark.parametrize('tiles', [1, 2, 3])
@pytest.mark.parametrize('M,N,K', [(64, 256, 64), (200, 300, 64), (1000, 700, 256), (513, 129, 37)])
def test_tensor_core_update_matches(M, N, K, tiles):
    """One tile a CTA (k_umma_update) and runs of 2 or 3 tiles a CTA with two accumulators (k_umma_runs, forced on
    these small updates: min_tiles 1), the last run short where the tile count does not divide."""
    from mom25d_b200 import _lib
    _lib.check(_lib.lib().m25_set_umma_tiles(tiles, 1))
    rng = np.random.default_rng(M + N + K)
    ld = max(M, K) + 3
    C = (rng.standard_normal((N, ld)) + 1j * rng.standard_normal((N, ld))).astype(np.complex64)   # columns
    L = (rng.standard_normal((K, ld)) + 1j * rng.standard_normal((K, ld))).astype(np.complex64)
    U = (rng.standard_normal((N, ld)) + 1j * rng.standard_normal((N, ld))).astype(np.complex64)
    Cm, Lm, Um = C[:, :M].T, L[:, :M].T, U[:, :K].T                     # M x N, M x K, K x N (column-major)
    want = Cm.astype(complex) - Lm.astype(complex) @ Um.astype(complex)
    dC, dL, dU = _lib.dev(C), _lib.dev(L), _lib.dev(U)
    nb = 64 << 20
    work = torch.empty(nb, dtype=torch.uint8, device='cuda')
    _lib.check(_lib.lib().m25_cgemm_update_tf32(_lib.P(dC), ctypes.c_long(ld), M, N, K, _lib.P(dL), _lib.P(dU),
                                                _lib.P(work), ctypes.c_size_t(nb), _lib.stream_ptr()))
    _lib.sync_check()
    _lib.check(_lib.lib().m25_set_umma_tiles(1, -1))
    got = dC.cpu().numpy()[:, :M].T
    err = np.abs(got - want).max() / np.abs(want).max()
    # 3xTF32 keeps FP32 accuracy (accumulation over 2K real terms in FP32: ~1e-5 at K = 256), where a single
    # TF32 product would be off by ~1e-3
    assert err < 1e-5, err
    assert np.array_equal(dC.cpu().numpy()[:, M:], C[:, M:])   # nothing outside the block written
