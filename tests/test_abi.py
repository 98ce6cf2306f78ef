"""The C ABI without a GPU: the library loads and exports every function include/mom25d_b200.h declares."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    out = []
    for h in os.listdir(os.path.join(ROOT, 'include')):
        if h.endswith('.h'):
            src = open(os.path.join(ROOT, 'include', h)).read()
            src = re.sub(r'/\*.*?\*/', '', src, flags=re.S)
            out += re.findall(r'\b(m25_[a-z0-9_]+)\s*\(', src)
    return sorted(set(out))


def test_library_exports_every_declared_symbol():
    from mom25d_b200 import build
    lib = ctypes.CDLL(build.build())
    names = declared()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    lib.m25_version.restype = ctypes.c_char_p
    assert b'sm_100a' in lib.m25_version()


def test_a_call_without_a_gpu_fails_loudly():
    """No CPU fallback: the device query reports a CUDA error (no device here), it does not pretend."""
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is present')
    from mom25d_b200 import _lib
    sms, free, total = ctypes.c_int(), ctypes.c_size_t(), ctypes.c_size_t()
    rc = _lib.lib().m25_device_info(ctypes.byref(sms), ctypes.byref(free), ctypes.byref(total))
    assert rc != 0 and _lib.lib().m25_last_error()
    with pytest.raises(_lib.M25Error):
        _lib.require_cuda()


def test_core_module_carries_the_reference_core_names():
    """mom25d_b200.core is a drop-in for fast.set_core (fast.py:27-51): every name the reference's direct solver and
    table builders call on its compiled core (fast.py, via.py, sim.py) exists here."""
    from mom25d_b200 import core
    for name in ('fill_far', 'fill_far_c64', 'far_block', 'matvec_far', 'matvec_far_multi', 'near_into_dense',
                 'near_coo', 'near_matvec', 'near_q', 'near_pairs', 'radial_table_sum', 'fan_q', 'hankel_real',
                 'bessel_jn_complex', 'scale_c64', 'num_threads'):
        assert callable(getattr(core, name)), name
    assert core.num_threads() >= 1


def test_seams_fail_loudly_without_a_gpu():
    import numpy as np
    import torch
    if torch.cuda.is_available():
        pytest.skip('a GPU is present')
    from mom25d_b200 import core, _lib
    from mom25d_b200.backend import CudaBackend, GPUUnavailable, register
    with pytest.raises(_lib.M25Error):
        core.bessel_jn_complex(0, np.ones(3, complex))
    with pytest.raises(GPUUnavailable):
        CudaBackend()

    class FakeGpuModule:                                      # the reference's registry, gpu.py:118
        _BACKENDS = {}
    register(FakeGpuModule)
    assert FakeGpuModule._BACKENDS['cuda'] is CudaBackend
