"""
mom25d_b200.sim - the caller of the hot path with the reference's signatures (mom25d sim.py:331, run.py:41):
Simulation(...).sparams(f) / .currents(f, E) / .excitation(), solved on one GPU by the device-resident direct
solver (operator.DirectSolver).

Differences from the reference's Simulation, all outside the hot path: meshes are built by this package's
Manhattan tensor mesher (board.py) from rectangles, not by the shapely mesher; ports are via ports or gap ports
(lumped); no wave ports, lumped elements, metal loss, frills, slots, quads or loop/tree basis.

Precision policy (fast.py:704-850, 1075-1084): 'double' (the drop-in, matches the reference's complex128 path),
'mixed' (complex64 fill and LU refined in double by GMRES), 'auto' (mixed above MIXED_MIN_N unknowns). A mixed
solve whose refinement does not converge is redone in double on the GPU, and frequencies up to MIXED_RETRY x that
one stay in double (the reference's rule; it falls back to its CPU, this build has none).
"""
import time

import numpy as np
import torch

from .board import Board, LayerStack, Via, ViaPort, GapPort, mesh_layers
from .geometry import Geometry
from .operator import DirectSolver, SolveFailed

MIXED_MIN_N = 3500       # sim.py:61
MIXED_RETRY = 1.25       # fast.py:252


class RunLog:
    """Stage timings and notes (multilayer.py:30-53)."""

    def __init__(self, verbose=False):
        self.verbose, self.records, self.notes = verbose, [], []

    def note(self, msg):
        self.notes.append(msg)
        if self.verbose:
            print('  ' + msg)

    def record(self, stage, seconds, detail=''):
        self.records.append((stage, seconds, detail))


class Simulation:
    """A board solved on the GPU. Either Simulation(stack, shapes, ports, vias, dmax=...) with shapes
    {interface: [rects]}, or Simulation.from_board(board)."""

    def __init__(self, stack=None, shapes=None, ports=(), vias=(), dmax=0.3e-3, w_ref=None, ncross=6, grade=1.0,
                 near_fac=5.0, solver='direct', precision='auto', gpu='auto', verbose=False, board=None, tf32=None,
                 lumped=(), metal=None):
        # lumped (extras.SeriesLumped) and metal (extras.Metal): the reference's sim.py:331-333 arguments, added
        # into Z as fast.py:628-641 does; a lumped element's cut line becomes a mesh line (sim.py:438)
        if board is None:
            if stack is None or shapes is None:
                raise ValueError("Simulation needs (stack, shapes) or board=")
            vias = list(vias) + [p.via for p in ports if isinstance(p, ViaPort) and p.via not in vias]
            lines = {}
            for el in lumped:                             # along x: the cut is the line x = c.x; along y: y = c.y
                xl, yl = lines.setdefault(el.layer, ([], []))
                if abs(el.lp.d[0]) >= abs(el.lp.d[1]):
                    xl.append(float(el.lp.c[0]))
                else:
                    yl.append(float(el.lp.c[1]))
            nodes, tris, tl = mesh_layers(stack, shapes, dmax, ncross=ncross, grade=grade, w_ref=w_ref, vias=vias,
                                          lines=lines)
            board = Board(stack, nodes, tris, tl, list(vias), list(ports), dmax, near_fac, 'simulation',
                          {k: list(v) for k, v in shapes.items()})
        if solver != 'direct':
            raise ValueError("solver: 'direct' (the dense fill + LU; the compressed solvers are not part of this build)")
        if gpu == 'off':
            raise ValueError("gpu='off': this build has no CPU path")
        self.board, self.log = board, RunLog(verbose)
        t = time.perf_counter()
        self.geo = Geometry(board, near_fac)
        self.Ne, self.Nv, self.N = self.geo.Ne, self.geo.Nv, self.geo.N
        self.ports = self.geo.ports
        self.precision = precision if precision != 'auto' else ('mixed' if self.N > MIXED_MIN_N else 'double')
        if tf32 is None:
            from . import umma_available
            tf32 = umma_available()
        self.fast = DirectSolver(self.geo, tf32=tf32)
        self.lumped, self.metal = list(lumped), metal
        if self.lumped or metal is not None:
            from .extras import ExtraBlocks
            self.fast.extras = ExtraBlocks(self.geo, self.lumped, metal)
        self.solver = 'direct'
        self.log.record('setup', time.perf_counter() - t, f"N={self.N}, {self.fast.dg.npairs} near pairs")

    @classmethod
    def from_board(cls, board, **kw):
        return cls(board=board, **kw)

    def excitation(self):
        return self.geo.excitation()

    def currents(self, f, E):
        """Basis currents for the excitation columns E (sim.py:1014-1031): a complex128 device tensor. A result that
        is not finite raises FloatingPointError (never NaN S-parameters)."""
        I = self._currents(f, E)
        if not bool(torch.isfinite(torch.view_as_real(I)).all()):
            raise FloatingPointError(f"mom25d_b200: the solve at {f / 1e9:.4g} GHz is not finite (N = {self.N})")
        return I

    def _currents(self, f, E):
        prec = self.precision
        t = time.perf_counter()
        try:
            I = self.fast.solve_direct(f, E, precision=prec)
        except SolveFailed as e:
            # the matrix-free mixed path (no room for a double Z): redone in double, and up to MIXED_RETRY x f
            self.log.note(f"WARNING {e} - solving in double precision up to {MIXED_RETRY * f / 1e9:.4g} GHz")
            self.fast.mixed_failed = max(self.fast.mixed_failed, f)
            I = self.fast.solve_direct(f, E, precision='double')
        for msg in self.fast.log:
            self.log.note(msg)
        self.fast.log.clear()
        self.log.record('solve', time.perf_counter() - t, f"{f / 1e9:.4g} GHz, {self.fast.last_path}, "
                                                          f"iters {self.fast.iters}")
        return I

    def port_rows(self):
        """The rows of I that the lumped ports read, with their weights (sim.py:997-1003)."""
        rows, wts, which = [], [], []
        for j, p in enumerate(self.ports):
            if isinstance(p, ViaPort):
                rows.append(self.Ne + self.geo._port_chain(p)); wts.append(p.sign); which.append(j)
            else:
                idx, sig = self.geo.gap_edges(p)
                rows += idx.tolist(); wts += (sig * self.geo.rwg.l[idx]).tolist(); which += [j] * len(idx)
        return np.array(rows), np.array(wts), np.array(which)

    def sparams(self, f, keep=False):
        """S at f (sim.py:1045-1092, lumped ports): the excitation copied to the device, the solve, the port
        currents gathered there and read back."""
        E = self.excitation()
        I = self.currents(f, E)
        rows, wts, which = self.port_rows()
        Ir = I[torch.as_tensor(rows, device=I.device)].cpu().numpy()          # the port rows only
        n = len(self.ports)
        Ip = np.zeros((n, I.shape[1]), complex)
        np.add.at(Ip, which, wts[:, None] * Ir)
        Ap, Bp = np.zeros((n, n), complex), np.zeros((n, n), complex)
        for i, p in enumerate(self.ports):
            Vp = np.eye(n)[i]
            Ap[i], Bp[i] = (Vp + p.zc * Ip[i]) / (2 * np.sqrt(p.zc)), (Vp - p.zc * Ip[i]) / (2 * np.sqrt(p.zc))
        S = Bp @ np.linalg.inv(Ap)
        self.last = dict(f=f, I=I if keep else None, A=Ap, B=Bp)
        return S

    def sweep(self, freqs):
        return np.array([self.sparams(f) for f in freqs])
