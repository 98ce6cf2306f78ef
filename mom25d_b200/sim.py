"""
mom25d_b200.sim - the caller of the hot path with the reference's signatures (mom25d sim.py:331, run.py:41):
Simulation(...).sparams(f) / .currents(f, E) / .excitation(), solved on one GPU by the device-resident direct
solver (operator.DirectSolver).

Differences from the reference's Simulation, all outside the hot path: meshes are built by this package's
Manhattan tensor mesher (board.py) from rectangles, not by the shapely mesher, so feeds and ports run along x or y;
ports are via ports, gap ports (lumped) or wave ports on a straight feed (LinePort), with series lumped elements
and conductor loss (extras.py); no differential ports, frills, slots, quad cells or loop/tree basis.

Precision policy (fast.py:704-850, 1075-1084): 'double' (the drop-in, matches the reference's complex128 path),
'mixed' (complex64 fill and LU refined in double by GMRES), 'auto' (mixed above MIXED_MIN_N unknowns). A mixed
solve whose refinement does not converge is redone in double on the GPU, and frequencies up to MIXED_RETRY x that
one stay in double (the reference's rule; it falls back to its CPU, this build has none).
"""
import time

import numpy as np
import torch

from .board import Board, LayerStack, Via, ViaPort, GapPort, LinePort, mesh_layers, port_lines
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
            # the cut lines of gap ports and lumped elements, a wave port's gap and sample cuts (sim.py:424-440)
            lines = port_lines(ports, lumped, dmax)
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

    def sparams(self, f, keep=False):
        """S at f (sim.py:1045-1092): the excitation copied to the device, the solve, the rows of the currents
        that the ports read gathered there and read back, the waves and S on the host (lumped ports' voltages and
        currents; wave ports' fitted feed waves, then the reciprocity balance)."""
        E = self.excitation()
        I = self.currents(f, E)
        rows = self.geo.port_rows()
        Ih = np.zeros((self.N, I.shape[1]), complex)
        Ih[rows] = I[torch.as_tensor(rows, device=I.device)].cpu().numpy()      # the port rows only
        info = {}
        S = self.geo.sparams_from_currents(Ih, f, info)
        self.last = dict(f=f, I=I if keep else None, **info)
        for name in info.get('low_span', []):
            self.log.note(f"WARNING {f / 1e9:.2f} GHz port {name}: its feed samples span less than 0.4 rad - wave "
                          f"separation unreliable (lengthen the straight feed or use a via / gap port)")
        return S

    def sweep(self, freqs):
        return np.array([self.sparams(f) for f in freqs])
