"""
mom25d_b200.run - S-parameters over a band (mom25d run.py:41-84 solve_band) with the same signature: adaptive by
default (afs.adaptive_sweep: a rational AAA model of S through as few solves as afs_tol allows, given on `points`
frequencies, or on `freq`), or linear=N equally spaced solves; S renormalised from each port's reference
impedance (zc, or zc_fn(f)) to zref.
"""
import time

import numpy as np


def renorm(S, zc, zref):
    """run.py:14-23: S from reference impedances zc to zref."""
    zc, n = np.asarray(zc, float), S.shape[0]
    zref = np.broadcast_to(np.asarray(zref, float), (n,))
    if np.allclose(zc, zref):
        return S
    I = np.eye(n)
    Z = np.diag(np.sqrt(zc)) @ (I + S) @ np.linalg.inv(I - S) @ np.diag(np.sqrt(zc))
    zn = np.diag(1 / np.sqrt(zref)) @ Z @ np.diag(1 / np.sqrt(zref))
    return (zn - I) @ np.linalg.inv(zn + I)


def out_refs(sim, z0):
    """The output reference impedance of each port (run.py:26-34): z0 (ohms, or {port name: ohms})."""
    out = []
    for p in sim.ports:
        out.append(z0.get(p.name, 50.0) if isinstance(z0, dict) else z0)
    return np.array(out, float)


def _zc(sim, f):
    return np.array([p.zc_fn(f) if getattr(p, 'zc_fn', None) else p.zc for p in sim.ports])


def solve_band(sim, fmin, fmax, points=401, zref=50.0, linear=None, afs_tol=2e-3, max_solves=40, log=print,
               keep_mid=False, progress=None, on_step=None, keep_at=(), freq=None):
    """(f, S (nf, n, n), info) of sim over fmin..fmax at zref (run.py:41-84). info: solves, seconds, zref, the
    solved frequencies, the port names, and the adaptive sweep's history (afs) and tolerance. keep_at: frequencies
    solved among the samples whose currents are kept in sim.kept; keep_mid: one more solve at mid-band, its
    currents kept in sim.last; progress(solves, at most, f) after each solve; on_step(entry) after each model of
    the adaptive sweep; freq: the frequencies the adaptive model is given on, in place of `points`."""
    t0, zr, done = time.time(), out_refs(sim, zref), []
    keep_at = {float(f) for f in keep_at}
    sim.kept = {}

    def solve(fr):
        if log:
            log(f"  solving {fr / 1e9:.4f} GHz")
        keep = float(fr) in keep_at
        S = renorm(sim.sparams(fr, keep=keep), _zc(sim, fr), zr)
        if keep:
            sim.kept[float(fr)] = sim.last['I']
        done.append(fr)
        if progress:
            progress(len(done), int(linear) if linear else max_solves, fr)
        return S
    if linear:
        fs = f = np.linspace(fmin, fmax, int(linear))
        S = np.array([solve(fi) for fi in f])
        hist = []
    else:
        from .afs import adaptive_sweep
        f, S, fs, _, hist = adaptive_sweep(solve, fmin, fmax, tol=afs_tol, ngrid=points, max_points=max_solves,
                                           log=log, on_step=on_step, seed=sorted(keep_at), grid=freq)
        if hist and not hist[-1].get('converged', True):
            sim.log.note(f"WARNING adaptive sweep: stopped at its {max_solves} solves before its models agreed (last "
                         f"change {hist[-1]['change']:.1e} at {hist[-1]['f_change'] / 1e9:.4g} GHz, tolerance "
                         f"{afs_tol:g}): more solves or a narrower band")
    if keep_mid:
        sim.sparams(fs[len(fs) // 2], keep=True)
    return f, S, dict(solves=len(fs), seconds=time.time() - t0, zref=zr.tolist(), solved=list(map(float, fs)),
                      names=[p.name for p in sim.ports], afs=hist, afs_tol=afs_tol)
