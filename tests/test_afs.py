"""The adaptive frequency sweep (afs.py: set-valued AAA after Nakatsukasa, Sete and Trefethen 2018) on the CPU,
with solves replaced by closed-form S-parameters: a rational response is recovered exactly; a line section with
a delay (not rational) is modelled within the tolerance over the whole grid; the solved frequencies' S are
returned exactly; a log-spaced grid is modelled in log f; non-finite S stops the sweep; max_points caps it."""
import numpy as np
import pytest

from mom25d_b200.afs import aaa, aaa_eval, adaptive_sweep


def line_section(f, tau=0.8e-9, r=0.3):
    e = np.exp(-2j * np.pi * f * tau)
    s11 = r * (1 - e ** 2) / (1 - r ** 2 * e ** 2)
    s21 = (1 - r ** 2) * e / (1 - r ** 2 * e ** 2)
    return np.array([[s11, s21], [s21, s11]])


def resonant(f):
    x = f / 1e9
    p = np.array([3.2 + 0.15j, 4.7 + 0.08j, 7.5 + 0.5j])
    s11 = 0.1 + 0.02j * np.sum(1 / (x - p))
    s21 = 0.8 + 0.01 * np.sum(np.array([1, -2, 0.5]) / (x - p))
    return np.array([[s11, s21], [s21, 0.9 * s11]])


def test_aaa_recovers_a_rational_function():
    z = np.linspace(1, 6, 30)
    F = np.array([resonant(x * 1e9).ravel() for x in z])
    sup, vals, w = aaa(z, F, tol=1e-13)
    x = np.linspace(1, 6, 301)
    ref = np.array([resonant(v * 1e9).ravel() for v in x])
    assert np.abs(aaa_eval(x, z[sup], vals, w) - ref).max() <= 1e-10
    assert len(sup) <= 8


@pytest.mark.parametrize('fn,tol', [(resonant, 2e-3), (line_section, 2e-3), (line_section, 1e-5)])
def test_adaptive_sweep_models_the_band(fn, tol):
    calls = []

    def solve(f):
        calls.append(f)
        return fn(f)
    fg, Sg, fs, Ss, hist = adaptive_sweep(solve, 1e9, 6e9, tol=tol, ngrid=401, log=None)
    true = np.array([fn(f) for f in fg])
    assert hist[-1]['converged']
    assert np.abs(Sg - true).max() <= tol
    assert len(fs) == len(calls) < 40 and np.array_equal(fs, np.sort(calls))
    for f, S in zip(fs, Ss):
        assert np.array_equal(S, fn(f))
    assert fg[0] == 1e9 and fg[-1] == 6e9 and len(fg) == 401


def test_adaptive_sweep_log_grid_and_caps():
    grid = np.geomspace(0.5e9, 10e9, 201)
    fg, Sg, fs, Ss, hist = adaptive_sweep(line_section, 0.5e9, 10e9, tol=2e-3, grid=grid, log=None)
    assert np.abs(Sg - np.array([line_section(f) for f in fg])).max() <= 2e-3
    fg, Sg, fs, Ss, hist = adaptive_sweep(line_section, 1e9, 6e9, tol=1e-12, max_points=9, log=None)
    assert len(fs) == 9 and not hist[-1]['converged']
    with pytest.raises(FloatingPointError):
        adaptive_sweep(lambda f: np.full((2, 2), np.nan), 1e9, 6e9, log=None)
