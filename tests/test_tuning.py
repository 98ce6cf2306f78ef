"""The LU's tuning table (m25_set_lu_tuning / m25_get_lu_tuning, filled by the autotuner mom25d_b200.tune): entry
lookup by size, the defaults without entries, argument checks, and the table file the library applies at load.
Host-side only: no kernel runs."""
import ctypes
import json

import pytest

from mom25d_b200 import _lib


def _get(L, n, single=1):
    a, b = ctypes.c_int(), ctypes.c_int()
    assert L.m25_get_lu_tuning(n, single, ctypes.byref(a), ctypes.byref(b)) == 0
    return a.value, b.value


def test_table_lookup_and_defaults(monkeypatch):
    monkeypatch.delenv('M25_NB2', raising=False)
    monkeypatch.delenv('M25_PANEL_BLOCKS', raising=False)
    from mom25d_b200 import tune
    L = _lib.lib()
    tune.set_table([(15000, 192, 48), (1000, 128, 16)])
    try:
        assert _get(L, 500) == (128, 16)                   # the entry nearest in log n
        assert _get(L, 3800) == (128, 16) and _get(L, 4000) == (192, 48)
        assert _get(L, 18788) == (192, 48)
        assert _get(L, 18788, single=0) == (256, min(32, _get(L, 18788, single=0)[1]))   # complex128: its own table
        monkeypatch.setenv('M25_NB2', '64')
        assert _get(L, 18788)[0] == 64                     # the environment overrides
        monkeypatch.delenv('M25_NB2')
        bad = (ctypes.c_int * 1)
        assert L.m25_set_lu_tuning(1, bad(5), bad(100), bad(3), 1) == 1   # nb2 not a multiple of 64
        assert _get(L, 18788) == (192, 48)                 # a refused table leaves the last one
    finally:
        tune.set_table([])
    nb2, blocks = _get(L, 5000)
    assert nb2 == 256 and 1 <= blocks <= 32


def test_tuning_file_is_applied(tmp_path):
    L = _lib.lib()
    f = tmp_path / 't.json'
    f.write_text(json.dumps(dict(device='test', sms=None, complex64=[dict(n=1, nb2=256, blocks=24, ms=1.0)],
                                 complex128=[dict(n=1, nb2=192, blocks=16, ms=1.0)])))
    try:
        assert _lib.apply_tuning(L, str(f))
        assert _get(L, 20000) == (256, 24) and _get(L, 20000, single=0) == (192, 16)
    finally:
        L.m25_set_lu_tuning(1, None, None, None, 0)
        L.m25_set_lu_tuning(0, None, None, None, 0)
        _lib.apply_tuning(L)                               # back to the committed table, if any
