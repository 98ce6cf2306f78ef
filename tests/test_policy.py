"""The mixed sweep's host-side policy, without a GPU: how many complex64 LUs stay kept (HBM-bounded, or the
reference's cap of 4), the reach learnt with the reference's rule (fast.py:989-994) over the attempts within half
an octave of f, the nearest kept factor within it, and the double band above a complex64 failure (the reference's
1.25 f, then the kept double factor's neighbourhood)."""
import numpy as np
import pytest

from mom25d_b200 import operator as OP


class _Geo:
    N = 18788


def solver(**kw):
    s = OP.DirectSolver.__new__(OP.DirectSolver)        # no device geometry: the policy alone
    s.geo, s.reuse, s.keep = _Geo(), True, kw.get('keep')
    s.kept, s.kept64 = [], None
    s.forget()
    return s


def test_keep_is_bounded_by_hbm_or_by_the_reference_cap(monkeypatch):
    GB = 1e9
    monkeypatch.setattr(OP.torch.cuda, 'mem_get_info', lambda: (150 * GB, 180 * GB))
    assert solver()._keep_max() == 16                    # KEEP_HBM's count (2.8 GB each, 40% of HBM: 25)
    assert solver(keep=4)._keep_max() == 4               # the reference's REUSE_KEEP
    monkeypatch.setattr(OP.torch.cuda, 'mem_get_info', lambda: (150 * GB, 40 * GB))
    assert solver()._keep_max() == int(0.4 * 40 * GB // (8.0 * 18788 ** 2))   # 40% of a smaller device
    monkeypatch.setattr(OP.torch.cuda, 'mem_get_info', lambda: (5 * GB, 180 * GB))
    assert solver()._keep_max() == 1                     # what is free: (0.9 x 5 GB - 0.4 GB) // 2.8 GB
    s = solver()
    s.reuse = False
    assert s._keep_max() == 0


def test_reach_replays_the_reference_rule_over_half_an_octave():
    s = solver()
    ln2 = np.log(2.0)
    assert s._reach_at(2e9) == pytest.approx(ln2)
    s._reach_learn(8.6e9, 0.45, False, [10], 26)         # a failure at 8.6 GHz narrows its own neighbourhood
    assert s._reach_at(8.0e9) == pytest.approx(0.8 * 0.45)
    assert s._reach_at(2.0e9) == pytest.approx(ln2)      # two octaves away: untouched
    s._reach_learn(6.38e9, 0.15, False, [10], 26)
    assert s._reach_at(6.0e9) == pytest.approx(0.8 * 0.15)
    s._reach_learn(1.93e9, 0.6, True, [9], 27)          # a quick success (<= cap / 2) widens to 1.25 d
    assert s._reach_at(2.0e9) == pytest.approx(1.25 * 0.6)
    s._reach_learn(2.6e9, 0.45, True, [25], 27)         # a slow success changes nothing
    assert s._reach_at(2.2e9) == pytest.approx(1.25 * 0.6)
    # the rule is replayed in order: a failure after a widening narrows again
    s._reach_learn(2.2e9, 0.5, False, [10], 27)
    assert s._reach_at(2.1e9) == pytest.approx(0.8 * 0.5)


def test_the_nearest_kept_factor_is_reused_within_the_local_reach():
    s = solver()
    s.kept = [(1.657e9, 'lu1', None, 0.2), (5.493e9, 'lu2', None, 0.2)]
    assert s._reusable(1.93e9)[1] == 'lu1'
    assert s._reusable(4.5e9)[1] == 'lu2'
    assert s._reusable(0.7e9) is None                    # 2.4x away: beyond ln 2
    s._reach_learn(6.38e9, 0.15, False, [10], 26)
    assert s._reusable(6.2e9) is None                    # 1.13x but the local reach is 0.12
    s.reuse = False
    assert s._reusable(1.93e9) is None


def test_double_band_above_a_complex64_failure():
    s = solver()
    assert not s._double_band(0.5e9)
    s.mixed_failed = 0.5e9
    assert s._double_band(0.6e9)                         # the reference's 1.25 f
    assert not s._double_band(0.78e9)                    # past it, without a kept double factor
    s.kept64 = (0.5e9, 'lu64', None, 0.7)
    assert s._double_band(0.78e9)                        # 1.57 f, the kept double factor within ln 1.6
    assert not s._double_band(0.85e9)                    # 1.7 f: past DOUBLE_UP
    s.kept64 = (0.45e9, 'lu64', None, 0.7)
    assert not s._double_band(0.78e9)                    # its kept factor 1.73x away
