"""
mom25d_b200._lib - the ctypes binding of libmom25d_b200.so (include/mom25d_b200.h). Device buffers are torch CUDA
tensors (PyTorch supplies memory and streams only); every call is checked and raises M25Error with the library's
message. There is no CPU fallback: without the library or a CUDA device the first call raises.
"""
import ctypes
import os

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libmom25d_b200.so')


class M25Error(RuntimeError):
    """An error reported by libmom25d_b200 (bad argument, CUDA error, or a kernel's own check)."""


class Mesh(ctypes.Structure):
    _fields_ = [('Ne', ctypes.c_int), ('Nt', ctypes.c_int)] + \
               [(n, ctypes.c_void_p) for n in ('ep', 'em', 'lt', 'te', 'ap', 'am', 'vp', 'vm', 'cent', 'area', 'ta',
                                               'tv')]


class Tables(ctypes.Structure):
    _fields_ = [('ntab', ctypes.c_int), ('nfine', ctypes.c_int), ('L', ctypes.c_int)] + \
               [(n, ctypes.c_void_p) for n in ('A', 'Q', 'cA', 'cq', 'cAi', 'cqi', 'dr', 'd', 'dimg', 'tab', 'kind')]


TablesF = Tables      # m25_tables_f: the same layout, complex64 / float32 arrays


class Quad(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ('nodes', 'tris', 'P3', 'W3', 'P6', 'W6')]


_lib = None
EXPORTS = ['m25_version', 'm25_last_error', 'm25_device_info', 'm25_spectral', 'm25_hankel', 'm25_spline_uniform',
           'm25_fill_far', 'm25_far_block', 'm25_near', 'm25_near_pairs', 'm25_fan_q', 'm25_radial_table_sum',
           'm25_matvec_far_multi', 'm25_equilibrate', 'm25_getrf_workspace', 'm25_getrf', 'm25_getrs',
           'm25_bessel_jn_complex']


def lib():
    """The loaded library (built in-tree by mom25d_b200.build); raises M25Error if it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise M25Error(f"libmom25d_b200.so is not built ({LIB_PATH}): python -m mom25d_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        L.m25_version.restype = ctypes.c_char_p
        L.m25_last_error.restype = ctypes.c_char_p
        L.m25_getrf_workspace.restype = ctypes.c_size_t
        L.m25_getrs_aux_bytes.restype = ctypes.c_size_t
        L.m25_getrf_workspace.argtypes = [ctypes.c_int, ctypes.c_int]
        L.m25_pair_record_bytes.restype = ctypes.c_size_t
        L.m25_launch_count.restype = ctypes.c_longlong
        _lib = L
        apply_tuning(L)
    return _lib


def apply_tuning(L, path=None):
    """The autotuner's LU parameters (tune.py, tuning_b200.json beside this file), where that file exists and was
    made on a device with this SM count; otherwise the library's defaults stay."""
    import json
    path = path or os.path.join(HERE, 'tuning_b200.json')
    if not os.path.exists(path):
        return False
    doc = json.load(open(path))
    try:
        if torch.cuda.is_available() and torch.cuda.get_device_properties(0).multi_processor_count != doc.get('sms'):
            return False
    except Exception:
        pass
    ok = True
    for single, key in ((1, 'complex64'), (0, 'complex128')):
        ent = doc.get(key, [])
        arr = lambda k: (ctypes.c_int * max(1, len(ent)))(*[int(e[k]) for e in ent])
        ok = L.m25_set_lu_tuning(single, arr('n'), arr('nb2'), arr('blocks'), len(ent)) == 0 and ok
    return ok


def check(rc, what=''):
    if rc != 0:
        msg = lib().m25_last_error().decode(errors='replace')
        raise M25Error(f"{what or 'libmom25d_b200'}: error {rc}: {msg}")


def require_cuda():
    if not torch.cuda.is_available():
        raise M25Error("no CUDA device: the hot path runs on the GPU only")


def P(t):
    """The device (or host) address of a tensor / array, for the C ABI."""
    if t is None:
        return ctypes.c_void_p(None)
    if isinstance(t, np.ndarray):
        return ctypes.c_void_p(t.ctypes.data)
    return ctypes.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def sync_check(stream=None, what='kernel'):
    check(lib().m25_sync_check(stream_ptr(stream)), what)


def dev(a, dtype=None):
    """A numpy array as a contiguous CUDA tensor."""
    a = np.ascontiguousarray(a if dtype is None else np.asarray(a, dtype))
    return torch.from_numpy(a).to('cuda', non_blocking=False)


def cview(t):
    """A complex CUDA tensor as its float view (interleaved re, im)."""
    return torch.view_as_real(t) if t.is_complex() else t
