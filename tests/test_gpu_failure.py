"""Failure detection on the GPU without a fault: every device wait in the library is bounded (the cooperative
kernels' grid barrier, the triangular solves' flags, the tensor-core pipeline's mbarriers) and, when its limit
runs out, writes M25_DEV_TIMEOUT to the device error word and lets the kernel return. Here the grid barrier is
entered by one block that waits for a second block which is never launched (m25_wait_selftest), so the wait runs
out by itself: m25_sync_check must report it, clear it, and the context must stay usable."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip('torch')


def test_a_bounded_wait_that_runs_out_is_reported_and_the_context_stays_usable():
    from mom25d_b200 import _lib
    L = _lib.lib()
    s = _lib.stream_ptr()
    assert L.m25_sync_check(s) == 0                            # nothing pending before
    assert L.m25_wait_selftest(s) == 0
    rc = L.m25_sync_check(s)
    assert rc == 4, rc                                          # M25_EDEVICE
    msg = L.m25_last_error().decode()
    assert '101' in msg and 'bounded wait gave up' in msg, msg
    assert L.m25_sync_check(s) == 0                             # reported once, then cleared
    # the context still works: a small factorisation and solve, checked against numpy
    n, k = 300, 2
    rng = np.random.default_rng(5)
    Z = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 3 * np.sqrt(n) * np.eye(n)
    Zd = _lib.dev(Z)
    ipiv = torch.empty(n, dtype=torch.int32, device='cuda')
    nb = int(L.m25_getrf_workspace(n, 0))
    work = torch.empty(nb, dtype=torch.uint8, device='cuda')
    _lib.check(L.m25_getrf(_lib.P(Zd), ctypes.c_long(n), n, _lib.P(ipiv), 0, 0, _lib.P(work), ctypes.c_size_t(nb), s),
               'm25_getrf')
    R = rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k))
    Rd = _lib.dev(R)
    _lib.check(L.m25_getrs(_lib.P(Zd), ctypes.c_long(n), n, _lib.P(ipiv), 0, _lib.P(Rd), k, s), 'm25_getrs')
    _lib.sync_check(what='solve after the timeout')
    X = Rd.cpu().numpy()
    # the factor is of Z^T (the reference's Fortran view, fast.py:318-358): its solve gives Z X = R
    assert np.abs(Z @ X - R).max() <= 1e-10 * np.abs(R).max()
