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
