"""
mom25d_b200.afs - the adaptive frequency sweep behind solve_band's default (the reference's run.py:66-75 calls
emsdev.afs.adaptive_sweep, from emsdev v0.3.1, which is not vendored with the reference, so its exact rules cannot
be read or pinned here). This one is built from the published method it names, AAA rational approximation
(Nakatsukasa, Sete and Trefethen, "The AAA algorithm for rational approximation", SIAM J. Sci. Comput. 40, 2018),
in its set-valued form (one set of support points and barycentric weights for all n^2 entries of S):

  1. solve a few frequencies spread over the band (both ends included, and any `seed` frequencies);
  2. fit the AAA model of S(f) through every frequency solved so far and evaluate it on the output grid;
  3. compare it with the previous model: the largest change over the grid and the frequency where it occurs;
  4. stop when that change has stayed at or below `tol` for two models in a row (or max_points solves were made);
     otherwise solve where the two models disagree most (never within a small distance of a solved frequency)
     and go back to 2.

On a band spanning more than a decade on a geometric grid, the model is a function of log f. The returned S on
the grid is the model's, with the solved S put back exactly where a grid point is a solved frequency.
"""
import numpy as np

SMALL = 1e-300


def aaa(z, F, tol=1e-13, mmax=100):
    """Set-valued AAA: support points (indices into z), their values and the barycentric weights of the rational
    r(x) = sum_s w_s F_s / (x - z_s) / sum_s w_s / (x - z_s) that fits F (m x p) at the points z (m,). Greedy: the
    next support point is the sample with the largest error, the weights the smallest right singular vector of
    the Loewner matrix of the remaining samples (stacked over the p columns); stops when every sample is within
    tol max|F| or mmax support points are used."""
    z = np.asarray(z, float)
    F = np.asarray(F, complex).reshape(len(z), -1)
    m = len(z)
    free = np.ones(m, bool)
    R = np.broadcast_to(F.mean(axis=0), F.shape).copy()
    scale = max(np.abs(F).max(), SMALL)
    sup, w = [], np.ones(1, complex)
    if m == 1:
        return np.array([0]), F[:1], w
    for _ in range(min(m - 1, mmax)):                     # (at least one sample stays a row of the Loewner matrix)
        err = np.abs(F - R).max(axis=1)
        err[~free] = -1.0
        j = int(np.argmax(err))
        sup.append(j)
        free[j] = False
        zs, fs = z[sup], F[sup]
        w = _weights(z, F, np.array(sup), free)
        C = 1.0 / (z[free, None] - zs[None, :])
        R = F.copy()
        R[free] = (C @ (w[:, None] * fs)) / (C @ w)[:, None]
        if np.abs(F - R).max() <= tol * scale:
            break
    return np.array(sup), F[sup], w


def _weights(z, F, sup, free):
    zs, fs = z[sup], F[sup]
    C = 1.0 / (z[free, None] - zs[None, :])                              # (r, k)
    L = (F[free][:, None, :] - fs[None, :, :]) * C[:, :, None]           # (r, k, p): Loewner, one block a column
    L = np.transpose(L, (0, 2, 1)).reshape(-1, len(sup))
    return np.linalg.svd(L, full_matrices=False)[2][-1].conj()


def aaa_eval(x, zs, fs, w):
    """The AAA model at the points x: (len(x), p); exact values at support points."""
    x = np.asarray(x, float)
    d = x[:, None] - zs[None, :]
    hit = np.abs(d) < 1e-14 * max(1.0, np.abs(zs).max())
    d[hit] = 1.0
    C = 1.0 / d
    out = (C @ (w[:, None] * fs)) / (C @ w)[:, None]
    rows, cols = np.nonzero(hit)
    out[rows] = fs[cols]
    return out


def _is_log(grid):
    g = np.asarray(grid, float)
    return len(g) > 2 and g[0] > 0 and g[-1] / g[0] > 10 and np.allclose(np.diff(np.log(g)), np.log(g[1] / g[0]),
                                                                         rtol=1e-6)


def adaptive_sweep(solve, fmin, fmax, tol=2e-3, ngrid=401, max_points=40, log=print, on_step=None, seed=(), grid=None,
                   n_start=5):
    """S over the band from as few solves as the tolerance allows. solve(f) -> S (n x n). Returns (f grid, S on the
    grid (nf, n, n), the solved frequencies (sorted), their S, history): history has one dict per model after the
    first, with the solves so far, the largest change from the previous model over the grid ('change'), where
    ('f_change') and 'converged'."""
    fgrid = np.asarray(grid, float) if grid is not None else np.linspace(fmin, fmax, int(ngrid))
    uselog = _is_log(fgrid)
    xf = (lambda f: np.log(np.asarray(f, float))) if uselog else (lambda f: np.asarray(f, float) / 1e9)
    xg = xf(fgrid)
    span = xg[-1] - xg[0]
    min_gap = 0.25 * span / max(len(fgrid) - 1, 1)
    start = xg[0] + span * 0.5 * (1 - np.cos(np.pi * np.arange(n_start) / (n_start - 1)))   # Chebyshev points
    todo = sorted(set(float(v) for v in np.interp(start, xg, fgrid)) | {float(f) for f in seed})
    solved = {}

    def take(f):
        S = np.asarray(solve(f), complex)
        if not np.all(np.isfinite(S)):
            raise FloatingPointError(f"adaptive sweep: the solve at {f / 1e9:.4g} GHz gave non-finite S-parameters")
        solved[float(f)] = S

    for f in todo:
        take(f)
    hist, prev, calm = [], None, 0
    while True:
        fs = np.array(sorted(solved))
        Ss = np.array([solved[f] for f in fs])
        n = Ss.shape[1]
        zs_i, vals, w = aaa(xf(fs), Ss.reshape(len(fs), -1), tol=1e-12)
        model = aaa_eval(xg, xf(fs)[zs_i], vals, w)
        if prev is not None:
            diff = np.abs(model - prev).max(axis=1)
            k = int(np.argmax(diff))
            change = float(diff[k])
            calm = calm + 1 if change <= tol else 0
            entry = dict(solves=len(fs), change=change, f_change=float(fgrid[k]), converged=calm >= 2)
            hist.append(entry)
            if log:
                log(f"  adaptive sweep: {len(fs)} solves, model change {change:.1e} at {fgrid[k] / 1e9:.4g} GHz")
            if on_step:
                on_step(entry)
            if calm >= 2:
                break
        if len(fs) >= max_points:
            if hist:
                hist[-1]['converged'] = False
            break
        # the next frequency: where the last two models differ most; before there are two, the widest gap's middle
        far = np.min(np.abs(xg[:, None] - xf(fs)[None, :]), axis=1) > min_gap
        if not far.any():
            break
        if prev is None:
            gaps = np.diff(xf(fs))
            i = int(np.argmax(gaps))
            f_next = float(np.interp(0.5 * (xf(fs)[i] + xf(fs)[i + 1]), xg, fgrid))
        else:
            score = np.where(far, np.abs(model - prev).max(axis=1), -1.0)
            f_next = float(fgrid[int(np.argmax(score))])
        prev = model
        take(f_next)
    out = model.reshape(len(fgrid), n, n)
    for f, S in solved.items():                           # the solved values, exactly, where they are on the grid
        hit = np.flatnonzero(np.abs(fgrid - f) <= 1e-9 * f)
        out[hit] = S
    fs = np.array(sorted(solved))
    return fgrid, out, fs, np.array([solved[f] for f in fs]), hist
