"""
mom25d_b200.run - S-parameters over a band (mom25d run.py:41-84 solve_band) with the same signature.
linear=N solves N equally spaced frequencies; the adaptive (AAA) sweep of the reference lives in its emsdev
dependency and is not part of this build: asking for it raises NotImplementedError.
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


def solve_band(sim, fmin, fmax, points=401, zref=50.0, linear=None, afs_tol=2e-3, max_solves=40, log=print,
               keep_mid=False, progress=None, on_step=None, keep_at=(), freq=None):
    """(f, S (nf, n, n), info) of sim over fmin..fmax at zref."""
    if not linear:
        raise NotImplementedError("the adaptive sweep (emsdev.afs) is not part of this build: pass linear=N")
    t0, done = time.time(), []
    zc = np.array([p.zc for p in sim.ports])
    f = np.linspace(fmin, fmax, int(linear))
    S = []
    for fi in f:
        log(f"  solving {fi / 1e9:.4f} GHz")
        S.append(renorm(sim.sparams(fi), zc, zref))
        done.append(fi)
        if progress:
            progress(len(done), int(linear), fi)
    return f, np.array(S), dict(solves=len(done), seconds=time.time() - t0, zref=np.broadcast_to(zref, len(zc)).tolist(),
                                solved=list(map(float, done)), names=[p.name for p in sim.ports], afs=[], afs_tol=afs_tol)
