"""m25_getrs_noalloc: the triangular solves of m25_getrs on fixed file-scope device scratch (no device allocation
during the call). Its results against m25_getrs on the same factor, on two calls in a row; sizes above the fixed
scratch rejected with a message. Collected last, so that it also runs after every other GPU test in one process."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip('torch')


def test_oversized_solve_is_rejected_before_any_device_work():
    from mom25d_b200 import _lib
    L = _lib.lib()
    L.m25_getrs_aux_bytes.restype = ctypes.c_size_t
    n = 30000
    assert L.m25_getrs_aux_bytes(n, 1) > (32 << 20)
    dummy = ctypes.c_void_p(256)                       # never dereferenced: the size check comes first
    rc = L.m25_getrs_noalloc(dummy, ctypes.c_long(n), n, dummy, 1, dummy, 2, None)
    assert rc == 1                                     # M25_EINVAL
    msg = L.m25_last_error().decode()
    assert 'm25_getrs_noalloc' in msg and 'scratch bytes' in msg


@pytest.mark.gpu
@pytest.mark.parametrize('single', [1, 0])
def test_noalloc_solves_match_getrs_twice(single):
    from mom25d_b200 import _lib
    L = _lib.lib()
    n, k = 1500, 3
    rng = np.random.default_rng(11)
    dt = np.complex64 if single else np.complex128
    Z = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 4 * np.sqrt(n) * np.eye(n)).astype(dt)
    Zd = _lib.dev(Z)
    ipiv = torch.empty(n, dtype=torch.int32, device='cuda')
    nb = int(L.m25_getrf_workspace(n, single))
    work = torch.empty(nb, dtype=torch.uint8, device='cuda')
    _lib.check(L.m25_getrf(_lib.P(Zd), ctypes.c_long(n), n, _lib.P(ipiv), single, 0, _lib.P(work),
                           ctypes.c_size_t(nb), _lib.stream_ptr()), 'm25_getrf')
    x = None
    for call in range(2):
        R = (rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k))).astype(dt)
        Ra, Rb = _lib.dev(R), _lib.dev(R)
        _lib.check(L.m25_getrs(_lib.P(Zd), ctypes.c_long(n), n, _lib.P(ipiv), single, _lib.P(Ra), k,
                               _lib.stream_ptr()), 'm25_getrs')
        _lib.check(L.m25_getrs_noalloc(_lib.P(Zd), ctypes.c_long(n), n, _lib.P(ipiv), single, _lib.P(Rb), k,
                                       _lib.stream_ptr()), 'm25_getrs_noalloc')
        _lib.sync_check(what='solves')
        a, b = Ra.cpu().numpy(), Rb.cpu().numpy()
        tol = 1e-5 if single else 1e-13
        assert np.abs(b - a).max() <= tol * np.abs(a).max(), call
        x = np.linalg.solve(Z.astype(complex), R.astype(complex))
        assert np.abs(b - x).max() <= (1e-4 if single else 1e-11) * np.abs(x).max(), call


def _pool_high_water(rt, pool):
    err, v = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemHigh)
    assert int(err) == 0
    return int(v)


@pytest.mark.gpu
def test_noalloc_solve_takes_no_device_memory():
    """The property the entry point exists for: the stream-ordered pool's high-water mark (reset before each call)
    moves for the allocating solve, m25_getrs, and stays where it was for m25_getrs_noalloc; torch's caching
    allocator sees no allocation during the no-alloc call either."""
    from cuda.bindings import driver as cu, runtime as rt
    from mom25d_b200 import _lib
    L = _lib.lib()
    n, k, single = 1200, 2, 1
    rng = np.random.default_rng(12)
    Z = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 4 * np.sqrt(n) * np.eye(n)).astype(np.complex64)
    Zd = _lib.dev(Z)
    ipiv = torch.empty(n, dtype=torch.int32, device='cuda')
    nb = int(L.m25_getrf_workspace(n, single))
    work = torch.empty(nb, dtype=torch.uint8, device='cuda')
    s = _lib.stream_ptr()
    _lib.check(L.m25_getrf(_lib.P(Zd), ctypes.c_long(n), n, _lib.P(ipiv), single, 0, _lib.P(work),
                           ctypes.c_size_t(nb), s), 'm25_getrf')
    R = _lib.dev((rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k))).astype(np.complex64))
    Rb = R.clone()
    # first call on this device: the no-alloc entry point's once-per-device set-up happens here
    _lib.check(L.m25_getrs_noalloc(_lib.P(Zd), ctypes.c_long(n), n, _lib.P(ipiv), single, _lib.P(Rb), k, s),
               'm25_getrs_noalloc')
    _lib.sync_check(what='first no-alloc solve')
    dev = torch.cuda.current_device()
    err, pool = rt.cudaDeviceGetMemPool(dev)
    assert int(err) == 0
    def reset():
        r = rt.cudaMemPoolSetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemHigh, cu.cuuint64_t(0))
        assert int(r[0] if isinstance(r, tuple) else r) == 0
    torch.cuda.synchronize()
    reset()
    base = _pool_high_water(rt, pool)
    Ra = R.clone()
    _lib.check(L.m25_getrs(_lib.P(Zd), ctypes.c_long(n), n, _lib.P(ipiv), single, _lib.P(Ra), k, s), 'm25_getrs')
    _lib.sync_check(what='allocating solve')
    assert _pool_high_water(rt, pool) > base             # the check sees an allocation when there is one
    torch.cuda.synchronize()
    reset()
    base = _pool_high_water(rt, pool)
    Rb = R.clone()
    torch.cuda.synchronize()
    allocs = torch.cuda.memory_stats().get('allocation.all.allocated', 0)
    _lib.check(L.m25_getrs_noalloc(_lib.P(Zd), ctypes.c_long(n), n, _lib.P(ipiv), single, _lib.P(Rb), k, s),
               'm25_getrs_noalloc')
    _lib.sync_check(what='no-alloc solve')
    assert _pool_high_water(rt, pool) == base
    assert torch.cuda.memory_stats().get('allocation.all.allocated', 0) == allocs
    a, b = Ra.cpu().numpy(), Rb.cpu().numpy()
    assert np.abs(b - a).max() <= 1e-5 * np.abs(a).max()
