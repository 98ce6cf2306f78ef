"""
mom25d_b200.ports - what turns the solved currents into S-parameters for wave ports (the reference's edge ports on
a straight feed, LinePort): the feed's propagation constant and its forward / backward waves fitted on the
currents through sample cuts (base.py:161-172), the ports' reciprocity balance (sim.py:1121-1143), and the line
characterisation that gives a feed's gamma and Zc from a centre-fed line (sim.py:1150-1180, line_char_xs).

The fits are host arithmetic on a few dozen currents per port (read back from the device); everything per
frequency that scales with the mesh stays on the GPU.
"""
import numpy as np

BALANCE_FLOOR = 1e-2      # sim.py:38: ports coupled by less than this (|S_ij S_ji|) keep their scales
FIT_SPAN = 0.4            # sim.py:37: rad the sample cuts must span for a fitted gamma to be trusted


def fit_gamma(Ik, step):
    """The propagation constant gamma of a feed from the currents Ik (n_cuts x columns) through equally spaced
    cuts `step` apart: on a uniform line I(s) = a exp(-gamma s) + b exp(gamma s), so that for three neighbouring
    cuts I_(k-1) + I_(k+1) = 2 cosh(gamma step) I_k whatever a and b are. cosh(gamma step) is taken as the least-
    squares solution of those relations over all interior cuts and columns; gamma is the branch with a
    non-negative real part (attenuation) and imaginary part (phase) - the role of the reference's fit_gamma."""
    Ik = np.asarray(Ik, complex)
    if Ik.ndim == 1:
        Ik = Ik[:, None]
    mid, sides = Ik[1:-1], Ik[:-2] + Ik[2:]
    x = np.vdot(mid, sides) / (2 * np.vdot(mid, mid).real)
    g = np.arccosh(x + 0j) / step
    return complex(abs(g.real), abs(g.imag))


def fit_waves(Ik, s, gamma):
    """The forward and backward wave amplitudes (a, b) per column with I(s) = a exp(-gamma s) + b exp(gamma s) at
    the cut positions s (relative to the reference plane), by least squares (the reference's fit_waves)."""
    s = np.asarray(s, float)
    basis = np.stack([np.exp(-gamma * s), np.exp(gamma * s)], axis=1)
    coef = np.linalg.lstsq(basis, np.asarray(Ik, complex), rcond=None)[0]
    return coef[0], coef[1]


def balance(S, exact=None, floor=BALANCE_FLOOR):
    """S made reciprocal, with the ports' scales (the reference's balance, sim.py:1121-1143). A wave port's two
    waves share the error of its reference impedance, so the computed S is D S_true D^-1 for a diagonal D: the
    transmissions S_ij and S_ji differ by d_i^2 / d_j^2 while the reflections and the products S_ij S_ji are
    right. log d is the weighted least-squares fit of log|S_ij / S_ji| / 2 = log d_i - log d_j over the port pairs,
    each pair weighted by |S_ij S_ji| (weak couplings carry little), every log d pulled toward 0 with the weight
    `floor` and the ports flagged in `exact` (lumped ones) held at 1; D is taken out and the rest of the asymmetry
    averaged."""
    A = np.abs(S)
    W = A * A.T
    np.fill_diagonal(W, 0.0)
    with np.errstate(divide='ignore', invalid='ignore'):
        half_log = np.where(W > 0, 0.5 * np.log(A / A.T), 0.0)
    L = np.diag(W.sum(axis=1) + floor) - W           # the normal equations: a graph Laplacian plus the hold
    if exact is not None and np.any(exact):
        L = L + np.diag(np.where(exact, 1e6, 0.0))
    d = np.exp(np.linalg.solve(L, (W * half_log).sum(axis=1)))
    S = S * (d[None, :] / d[:, None])
    return 0.5 * (S + S.T), d


def wave_port_waves(p, samples, Ik, f):
    """(A row, B row, gamma, fit residual, span) of wave port p: gamma known (p.gamma_fn) or fitted, the waves at
    the reference plane, A = sqrt(zc) cs a, B = -sqrt(zc) cs b (sim.py:1050-1075)."""
    gk = getattr(p, 'gamma_fn', None)
    step = abs(samples[1] - samples[0]) if len(samples) > 1 else 1.0
    g = gk(f) if gk is not None else fit_gamma(Ik, step)
    x = samples - p.ref
    a, b = fit_waves(Ik, x, g)
    model = np.stack([np.exp(-g * x), np.exp(g * x)], 1) @ np.vstack([a, b])
    resid = float(np.max(np.linalg.norm(Ik - model, axis=0)) / np.max(np.linalg.norm(Ik, axis=0)))
    cs = getattr(p, 'cscale', 1.0)
    span = abs(complex(g).imag) * abs(samples[-1] - samples[0])
    return np.sqrt(p.zc) * cs * a, -np.sqrt(p.zc) * cs * b, complex(g), resid, span


def line_char_xs(stack, layer, w, freqs, planes=None, coplanar=None, via_pitch=1e-3, via_r=0.15e-3, length=16e-3,
                 dmax=0.4e-3, ncross=4, verbose=False, precision='double'):
    """(gamma, Zc) over `freqs` of a strip of width w on interface `layer` (the reference's line_char_xs,
    sim.py:1150-1180): a centre-fed line `length` long with a wave port's sample cuts on each half, solved on the
    GPU; gamma fitted on both halves' cuts together, the waves of each half at the feed, Zc = 1 / (the net current
    the unit gap voltage drives). planes {interface: width}: a wide centred strip there (a meshed ground);
    coplanar [(y0, y1), ...]: grounded strips beside it on the same interface, a via row to the ground every
    via_pitch along their inner edge."""
    from .board import LinePort, Via
    from .sim import Simulation
    L2, margin = length / 2, 2e-3
    shapes = {layer: [(-L2, -w / 2, L2, w / 2)]}
    for k, W in (planes or {}).items():
        shapes.setdefault(k, []).append((-L2, -W / 2, L2, W / 2))
    vias = []
    for y0, y1 in (coplanar or []):
        shapes[layer].append((-L2, y0, L2, y1))
        inner = y0 if abs(y0) < abs(y1) else y1
        yv = inner + np.sign(y1 + y0) * min(0.5 * abs(y1 - y0), max(2 * via_r, 0.4e-3))
        vias += [Via(x, yv, 0, layer, radius=via_r, name='fence') for x in np.arange(-L2 + via_pitch / 2, L2, via_pitch)]
    step = max(dmax, (L2 - margin - 1e-3) / 8)            # a well-conditioned fit at low frequency
    ports = [LinePort(layer, (0, 0), (sgn, 0), w, L2 - margin, s0=1e-3, step=step, name=nm)
             for sgn, nm in ((1, 'R'), (-1, 'L'))]
    wr = {layer: w, **{k: min(W, 2e-3) for k, W in (planes or {}).items() if k != layer}}
    sim = Simulation(stack, shapes, ports, vias=vias, dmax=dmax, w_ref=wr, ncross=ncross, verbose=verbose,
                     precision=precision)
    geo = sim.geo
    gam, zc = [], []
    for f in freqs:
        I = sim.currents(f, geo.excitation()[:, [0]]).cpu().numpy()
        IR, IL = geo.cut_currents(I, 0), geo.cut_currents(I, 1)
        g = fit_gamma(np.hstack([IR, IL]), step)
        (A, B), (C, D) = fit_waves(IR, geo.samples[0], g), fit_waves(IL, geo.samples[1], g)
        gam.append(g)
        zc.append(1.0 / ((A[0] - B[0]) - (C[0] - D[0])))
    return np.array(gam), np.array(zc)
