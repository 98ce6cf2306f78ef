"""
mom25d_b200.board - the inputs of the per-frequency hot path: the layer stack, a Manhattan mesher, the RWG basis,
via chains and their fans, ports, and the packed geometry the fill kernels read.

Everything here runs once per board (mesh set-up), on the host, and produces plain arrays. The layouts follow the
reference's so that its kernels and ours read the same numbers:

  * LayerStack: interfaces 0..N, interface 0 the PEC ground at z = 0 (mom25d multilayer.py:90-250).
  * tensor_mesh: the non-uniform tensor mesher (multilayer.py:322-349), node numbering in order of first use.
  * RWG: interior edges in order of first appearance, T+ the first triangle of an edge (base.py:16-47).
  * pack_geometry: the compiled core's `g` and `q` dictionaries (fast.py:377-406).
  * routed_board: a seeded synthetic routed board (Manhattan traces, vias, edge ports), each trace run meshed by
    tensor_mesh on its own, so traces never share nodes.
"""
from dataclasses import dataclass, field

import numpy as np

MU0 = 4e-7 * np.pi
C0 = 299792458.0
EPS0 = 1.0 / (MU0 * C0 ** 2)


# ---- stack --------------------------------------------------------------------------------------------------------
class Layer:
    """A dielectric layer: thickness h (m), relative permittivity er and loss tangent tand (constant over f)."""

    def __init__(self, h, er, tand=0.0, name=None):
        self.h, self.er, self.tand, self.name = float(h), float(er), float(tand), name

    @property
    def er_c(self):
        return self.er * (1 - 1j * self.tand)


def check_stack(stack):
    """Raises NotImplementedError for a stack the device Green network does not model: an open bottom, PEC planes
    inside the stack, or layers whose permittivity depends on f (the reference's LayerStack(bottom='open',
    bottom_er, pec=(...)) and Layer(fref=...), multilayer.py:96-111, 118-127). Takes this module's LayerStack or
    the reference's own, so that such a stack is refused at the seam instead of solved as a grounded one."""
    bottom = getattr(stack, 'bottom', 'pec')
    planes = tuple(getattr(stack, 'pec', ()) or ())
    if bottom != 'pec':
        raise NotImplementedError("the layer stack has an open bottom (bottom=%r): the device Green network models "
                                  "a PEC ground at z = 0 only" % (bottom,))
    if planes:
        raise NotImplementedError("the layer stack has PEC planes at interfaces %s: the device Green network models "
                                  "no planes inside the stack" % (list(planes),))
    if getattr(stack, 'dispersive', False):
        raise NotImplementedError("the layer stack has wideband (frequency-dependent) layers: the device Green "
                                  "network takes constant permittivities")


class LayerStack:
    """Dielectric layers bottom -> top over a PEC ground (interface 0, z = 0); interface k is the top of layer k.
    top: 'open' (a half-space of top_er above) or 'pec' (a cover on interface N). Mirrors multilayer.py:90-250
    for grounded stacks: the reference's bottom='open' and internal PEC planes (pec=...) are accepted as arguments
    and refused with NotImplementedError (check_stack)."""

    def __init__(self, layers, top='open', top_er=1.0, bottom='pec', bottom_er=1.0, pec=()):
        if top not in ('open', 'pec'):
            raise ValueError("top: 'open' or 'pec'")
        if bottom not in ('open', 'pec'):
            raise ValueError("bottom: 'open' or 'pec'")
        self.layers, self.top, self.top_er = list(layers), top, float(top_er)
        self.N = len(self.layers)
        self.bottom, self.bottom_er = bottom, float(bottom_er)
        self.pec = tuple(sorted({int(k) for k in pec}))
        check_stack(self)
        self.z = np.concatenate([[0.0], np.cumsum([l.h for l in self.layers])])

    def eps(self, j):
        if 1 <= j <= self.N:
            return self.layers[j - 1].er_c
        return complex(1.0 if j <= 0 else self.top_er)

    def eps_sum(self, k):
        return self.eps(k) + self.eps(k + 1)

    def is_pec(self, k):
        return k == 0 or (k == self.N and self.top == 'pec')

    @property
    def metal_interfaces(self):
        return list(range(1, self.N + 1 if self.top == 'open' else self.N))

    @property
    def hmin(self):
        return min(l.h for l in self.layers)

    def max_er(self):
        return max([abs(l.er_c) for l in self.layers] + ([abs(self.top_er)] if self.top == 'open' else []))

    def nearest_discontinuity(self, k):
        """How far interface k is from the nearest interface, below or above it, where the permittivity steps or
        a PEC lies (the image term's reach, multilayer.py:170-176); inf where there is none."""
        def steps(j):
            return self.is_pec(j) or self.eps(j) != self.eps(j + 1)
        gaps = [abs(self.z[k] - self.z[j]) for j in range(self.N + 1) if j != k and steps(j)]
        return min(gaps, default=np.inf)


# ---- mesher -------------------------------------------------------------------------------------------------------
def graded(u, grade):
    """Positions u in [0, 1] pulled toward both ends by a cosine (grade 0: uniform, 1: fully cosine), the
    reference's cell grading across a strip (base.py:80-82)."""
    return (1 - grade) * u + grade * (1 - np.cos(np.pi * u)) / 2


def _axis_lines(edge_vals, port_vals, dmax, ncross, narrow, grade=0.0):
    """Grid coordinates along one axis, the same numbers as the reference's axis lines (multilayer.py:321-335):
    the distinct conductor-edge coordinates; between two neighbours at most `narrow` apart with no line to keep
    strictly inside them (a strip across its width), ncross cells graded toward both ends; every other interval
    is split at the lines to keep (ports, vias, cut lines) and each piece cut evenly into cells of at most dmax."""
    edges = np.unique(np.round(np.asarray(edge_vals, float), 12))
    pins = np.unique(np.round(np.asarray(port_vals, float), 12))
    pieces = [edges[:1]]
    for lo, hi in zip(edges[:-1], edges[1:]):
        inside = pins[(pins > lo + 1e-9) & (pins < hi - 1e-9)]
        if inside.size == 0 and hi - lo <= narrow + 1e-12:
            pieces.append(lo + (hi - lo) * graded(np.linspace(0, 1, ncross + 1)[1:], grade))
            continue
        stops = np.concatenate([[lo], inside, [hi]])
        for c, d in zip(stops[:-1], stops[1:]):
            cells = max(1, int(np.ceil((d - c) / dmax - 1e-9)))
            pieces.append(np.linspace(c, d, cells + 1)[1:])
    return np.concatenate(pieces)


def tensor_mesh(rects, dmax, ncross, narrow, xlines=(), ylines=(), grade=1.0):
    """multilayer.py:338-349: the union of axis-aligned rectangles on a tensor grid, each cell two triangles with
    alternating diagonals; nodes numbered in order of first use. Returns (nodes (n, 2), tris (m, 3))."""
    X, Y = (_axis_lines([r[a] for r in rects] + [r[a + 2] for r in rects], ls, dmax, ncross, narrow, grade)
            for a, ls in ((0, xlines), (1, ylines)))
    cx, cy = 0.5 * (X[:-1] + X[1:]), 0.5 * (Y[:-1] + Y[1:])
    inside = np.zeros((len(cx), len(cy)), bool)
    for x0, y0, x1, y1 in rects:
        inside |= ((cx[:, None] > x0) & (cx[:, None] < x1) & (cy[None, :] > y0) & (cy[None, :] < y1))
    I, J = np.nonzero(inside)                                   # row-major order, as np.nonzero gives it
    even = (I + J) % 2 == 0
    # the 4 corners of each cell; each cell's 2 triangles as corner indices
    corners = np.stack([np.stack([I, J], 1), np.stack([I + 1, J], 1), np.stack([I + 1, J + 1], 1),
                        np.stack([I, J + 1], 1)], 1)            # (ncell, 4, 2)
    keys = corners[..., 0] * (len(Y) + 1) + corners[..., 1]     # (ncell, 4)
    # node ids in order of first use: the corner order n0, n1, n2, n3 per cell (setdefault order)
    flat = keys.ravel()
    uniq, first = np.unique(flat, return_index=True)
    order = np.argsort(first, kind='stable')
    node_id = np.empty(len(uniq), np.int64)
    node_id[order] = np.arange(len(uniq))
    nid = node_id[np.searchsorted(uniq, keys)]                  # (ncell, 4)
    t_even = np.stack([nid[:, [0, 1, 2]], nid[:, [0, 2, 3]]], 1)
    t_odd = np.stack([nid[:, [0, 1, 3]], nid[:, [1, 2, 3]]], 1)
    tris = np.where(even[:, None, None], t_even, t_odd).reshape(-1, 3)
    ij = uniq[order]
    nodes = np.stack([X[ij // (len(Y) + 1)], Y[ij % (len(Y) + 1)]], 1)
    return nodes, tris


# ---- RWG basis ----------------------------------------------------------------------------------------------------
class RWG:
    """base.py:16-47: RWG functions on the interior edges (edges shared by two triangles), in order of first
    appearance; T+ the first triangle of the edge, vp / vm the free vertices, l the length, nrm the direction of
    positive current (T+ -> T-)."""

    def __init__(self, nodes, tris):
        self.nodes, self.tris = np.asarray(nodes, float), np.asarray(tris, np.int64)
        V = self.nodes[self.tris]
        e1, e2 = V[:, 1] - V[:, 0], V[:, 2] - V[:, 0]
        self.area = 0.5 * (e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0])
        if not (self.area > 0).all():
            raise ValueError("triangles must be counter-clockwise")
        self.cent = V.mean(1)
        Nt = len(self.tris)
        a, b, c = self.tris.T
        u = np.stack([a, b, c], 1).ravel()                      # the (t, i) slots in traversal order
        v = np.stack([b, c, a], 1).ravel()
        lo, hi = np.minimum(u, v), np.maximum(u, v)
        key = lo * (len(self.nodes) + 1) + hi
        uk, first, inv, cnt = np.unique(key, return_index=True, return_inverse=True, return_counts=True)
        if (cnt > 2).any():
            raise ValueError("an edge shared by more than two triangles")
        # second occurrence of each key: the last slot with that key
        last = np.empty(len(uk), np.int64)
        last[inv] = np.arange(len(key))
        sel = np.flatnonzero(cnt == 2)
        sel = sel[np.argsort(first[sel], kind='stable')]       # dict insertion order = first appearance
        s1, s2 = first[sel], last[sel]
        t1, i1, t2, i2 = s1 // 3, s1 % 3, s2 // 3, s2 % 3
        self.Ne = Ne = len(sel)
        self.tp, self.tm = t1, t2
        self.vp = self.nodes[self.tris[t1, (i1 + 2) % 3]]
        self.vm = self.nodes[self.tris[t2, (i2 + 2) % 3]]
        pu, pv = self.nodes[lo[s1]], self.nodes[hi[s1]]
        self.l = np.linalg.norm(pv - pu, axis=1)
        self.mid, self.ends = 0.5 * (pu + pv), np.stack([pu, pv], 1)
        tau = (pv - pu) / self.l[:, None]
        n = np.c_[tau[:, 1], -tau[:, 0]]
        n[((self.cent[t2] - self.cent[t1]) * n).sum(1) < 0] *= -1
        self.nrm = n
        self.Nt = Nt


# ---- quadrature rules (base.py:70-77) -----------------------------------------------------------------------------
_a1, _a2 = 0.445948490915965, 0.091576213509771
BAR6 = np.array([[1 - 2 * _a1, _a1, _a1], [_a1, 1 - 2 * _a1, _a1], [_a1, _a1, 1 - 2 * _a1],
                 [1 - 2 * _a2, _a2, _a2], [_a2, 1 - 2 * _a2, _a2], [_a2, _a2, 1 - 2 * _a2]])
W6 = np.array([0.223381589678011] * 3 + [0.109951743655322] * 3)
BAR3 = np.array([[2 / 3, 1 / 6, 1 / 6], [1 / 6, 2 / 3, 1 / 6], [1 / 6, 1 / 6, 2 / 3]])
W3 = np.ones(3) / 3


def quad_pts(rwg, bar):
    return np.einsum('qk,tkc->tqc', bar, rwg.nodes[rwg.tris])


# ---- vias and ports -----------------------------------------------------------------------------------------------
class Via:
    """A plated via on the axis (x, y) from interface k_bot to k_top with barrel radius `radius` (sim.py:154-160)."""

    def __init__(self, x, y, k_bot, k_top, radius=0.15e-3, name=''):
        self.x, self.y, self.k_bot, self.k_top, self.a, self.name = float(x), float(y), int(k_bot), int(k_top), \
            float(radius), name
        self.Z = None


class ViaPort:
    """A lumped port in a via's lowest chain, EMF + toward the top (sim.py:178-186)."""
    kind = 'via'

    def __init__(self, via, z0=50.0, name='', sign=1):
        self.via, self.zc, self.name, self.sign = via, float(z0), name, float(sign)


class GapPort:
    """A delta-gap port across a strip at `center`, `direction` along the strip, of width `width` (sim.py:163-175):
    the edges lying on the transverse line carry the EMF."""
    kind = 'gap'

    def __init__(self, layer, center, direction, width, z0=50.0, name=''):
        d = np.asarray(direction, float)
        self.layer, self.c, self.d = int(layer), np.asarray(center, float), d / np.linalg.norm(d)
        self.t = np.array([-self.d[1], self.d[0]])
        self.w, self.zc, self.name = float(width), float(z0), name


class LinePort:
    """A wave port on a straight feed (the reference's geo.LinePort, geo.py:24-56): a delta-gap source across the
    feed at `center`, `direction` pointing into the device along the feed, `width` the feed's width (the gap and
    the sample cuts span it); the reference plane `ref_dist` from the gap along the feed; sample cuts from s0 to s1
    every `step` (defaults 2 step, ref_dist and dmax), on which the forward and backward waves of the feed are fitted.
    zc: the reference impedance (zc_fn(f), where set, replaces it at each frequency); gamma_fn(f): a known
    propagation constant of the feed (from a line characterisation) used instead of fitting one."""
    kind = 'wave'

    def __init__(self, layer, center, direction, width, ref_dist, s0=None, step=None, zc=50.0, name='', s1=None):
        d = np.asarray(direction, float)
        self.layer, self.c, self.d = int(layer), np.asarray(center, float), d / np.linalg.norm(d)
        self.t = np.array([-self.d[1], self.d[0]])
        self.w, self.ref, self.s0, self.step, self.s1 = float(width), float(ref_dist), s0, step, s1
        self.zc, self.name = float(zc), name
        self.zc_fn = self.gamma_fn = None

    def line(self, s):
        """The ends of the transverse line at distance s from the gap along the feed."""
        p = self.c + self.d * s
        return p - self.t * self.w / 2, p + self.t * self.w / 2

    @property
    def axis_aligned(self):
        return abs(self.d[0]) < 1e-12 or abs(self.d[1]) < 1e-12

    def sample_positions(self, dmax):
        """The sample cuts' distances from the gap (sim.py:426-431): s1, s1 - step, ... down to no closer than s0,
        in increasing order."""
        step = self.step or dmax
        s0 = 2 * step if self.s0 is None else self.s0
        s1 = self.ref if self.s1 is None else self.s1
        count = int(np.floor((s1 - s0) / step + 1e-9)) + 1
        return s1 - step * np.arange(count)[::-1]


def port_lines(ports, lumped, dmax):
    """{interface: (x lines, y lines)}: the mesh lines the ports and lumped elements need (sim.py:424-440): a gap
    port's and a lumped element's cut, a wave port's gap and every sample cut. Axis-aligned feeds only (the
    tensor mesher)."""
    lines = {}

    def add(lp, at):
        if not (abs(lp.d[0]) < 1e-12 or abs(lp.d[1]) < 1e-12):
            raise ValueError("ports and lumped elements on the tensor mesh run along x or y")
        xs, ys = lines.setdefault(lp.layer, ([], []))
        along_x = abs(lp.d[0]) > 0.5
        for s in at:
            (xs if along_x else ys).append(float((lp.c + lp.d * s)[0 if along_x else 1]))
    for p in ports:
        if isinstance(p, LinePort):
            add(p, np.append(p.sample_positions(dmax), 0.0))
        elif isinstance(p, GapPort):
            add(p, [0.0])
    for el in lumped:
        add(el.lp, [0.0])
    return lines


@dataclass
class Board:
    """A meshed board: stack, mesh with each triangle's interface, vias, ports, and the mesh parameters."""
    stack: LayerStack
    nodes: np.ndarray
    tris: np.ndarray
    tri_layer: np.ndarray
    vias: list = field(default_factory=list)
    ports: list = field(default_factory=list)
    dmax: float = 0.3e-3
    near_fac: float = 5.0
    name: str = 'board'
    rects: dict = field(default_factory=dict)     # interface -> [(x0, y0, x1, y1)]: the copper, for on-metal tests

    def __post_init__(self):
        check_stack(self.stack)


def _on_copper(rects, x, y, tol=1e-9):
    return any(x0 - tol <= x <= x1 + tol and y0 - tol <= y <= y1 + tol for x0, y0, x1, y1 in rects)


def mesh_layers(stack, shapes, dmax, ncross=6, grade=1.0, w_ref=None, vias=(), pieces=None, lines=None):
    """The meshes of every interface of `shapes` ({interface: [rects]}) by tensor_mesh, concatenated in interface
    order. pieces ({interface: [[rects], ...]}): mesh each group of rectangles on its own (disjoint traces).
    Via axes on an interface become grid lines there, so each via has a mesh vertex on every interface it
    attaches to; lines ({interface: (xs, ys)}) adds grid lines (a lumped element's cut line).
    Returns (nodes, tris, tri_layer)."""
    nodes, tris, tl, off = [], [], [], 0
    for k in sorted(shapes):
        groups = (pieces or {}).get(k) or [shapes[k]]
        for rects in groups:
            vx = [v.x for v in vias if v.k_bot <= k <= v.k_top and _on_copper(rects, v.x, v.y)]
            vy = [v.y for v in vias if v.k_bot <= k <= v.k_top and _on_copper(rects, v.x, v.y)]
            lx, ly = (lines or {}).get(k, ((), ()))
            vx, vy = vx + list(lx), vy + list(ly)
            wr = w_ref.get(k) if isinstance(w_ref, dict) else w_ref
            nd, tr = tensor_mesh(rects, dmax, ncross, 1.01 * max(wr or 0, 1.5 * dmax), vx, vy, grade=grade)
            nodes.append(nd)
            tris.append(tr + off)
            tl.append(np.full(len(tr), k))
            off += len(nd)
    return np.vstack(nodes), np.vstack(tris), np.concatenate(tl)


# ---- the synthetic boards -----------------------------------------------------------------------------------------
def microstrip_board(dmax=0.3e-3, length=30e-3, width=3.0e-3, ports='via'):
    """A 2-port microstrip through line: one layer h = 1.6 mm, er = 4.4, tan d = 0.02 over the ground; a
    width x length strip on interface 1 centred at the origin; a via port from the ground to each strip end."""
    st = LayerStack([Layer(1.6e-3, 4.4, 0.02)])
    L2, w2 = length / 2, width / 2
    rects = {1: [(-L2, -w2, L2, w2)]}
    x_end = L2 - dmax / 2
    vias = [Via(-x_end, 0.0, 0, 1, 0.15e-3, 'P1'), Via(x_end, 0.0, 0, 1, 0.15e-3, 'P2')]
    nodes, tris, tl = mesh_layers(st, rects, dmax, vias=vias)
    return Board(st, nodes, tris, tl, vias, [ViaPort(v, 50.0, v.name) for v in vias], dmax, 5.0, 'microstrip',
                 rects)


def quarter_wave_length(f0, width, h, er):
    """Open-stub length c / (4 f0 sqrt(eps_eff)), eps_eff from Hammerstad's microstrip formula."""
    u = width / h
    eeff = (er + 1) / 2 + (er - 1) / 2 / np.sqrt(1 + 12 / u)
    return C0 / (4 * f0 * np.sqrt(eeff))


def stub_filter_board(dmax=0.2e-3, f0=2.4e9, width=1.1e-3, length=40e-3):
    """The stub notch filter: 3 layers h = 0.2 / 1.0 / 0.2 mm, er = 3.5 / 4.4 / 3.5, tan d = 0.02; a 50 ohm line
    width x length on the top (interface 3) and an open quarter-wave stub at f0 teed off at its midpoint (length
    from Hammerstad's eps_eff over the whole 1.4 mm dielectric); a via port from the ground at each line end."""
    st = LayerStack([Layer(0.2e-3, 3.5, 0.02), Layer(1.0e-3, 4.4, 0.02), Layer(0.2e-3, 3.5, 0.02)])
    h = float(st.z[-1])
    er = float(np.average([l.er for l in st.layers], weights=[l.h for l in st.layers]))
    Ls = quarter_wave_length(f0, width, h, er)
    L2, w2 = length / 2, width / 2
    rects = {3: [(-L2, -w2, L2, w2), (-w2, w2, w2, w2 + Ls)]}
    x_end = L2 - dmax / 2
    vias = [Via(-x_end, 0.0, 0, 3, 0.15e-3, 'P1'), Via(x_end, 0.0, 0, 3, 0.15e-3, 'P2')]
    nodes, tris, tl = mesh_layers(st, rects, dmax, w_ref={3: width}, vias=vias)
    return Board(st, nodes, tris, tl, vias, [ViaPort(v, 50.0, v.name) for v in vias], dmax, 5.0, 'stub_filter',
                 rects)


def routed_board(seed=0, n_traces=24, n_vias=16, n_ports=8, size=(60e-3, 40e-3), dmax=0.25e-3, ncross=3,
                 width=(0.15e-3, 0.5e-3), segments=(2, 5), seg_len=(3e-3, 20e-3), clearance=0.3e-3):
    """A seeded synthetic routed board on the stub filter's stack: n_traces Manhattan traces (width U[width],
    segments U{segments}, each U[seg_len] long, alternating x / y), each on the top (3) or the inner (1) copper
    interface at random; n_vias vias (radius 0.15 mm) at segment ends where a trace changes interface; n_ports
    via ports from the ground at the ends of the first n_ports / 2 traces. Traces on one interface keep
    `clearance` apart (no shorts). Each trace run is meshed on its own (tensor_mesh, ncross cells across)."""
    rng = np.random.default_rng(seed)
    st = LayerStack([Layer(0.2e-3, 3.5, 0.02), Layer(1.0e-3, 4.4, 0.02), Layer(0.2e-3, 3.5, 0.02)])
    W, H = size
    placed = {1: [], 3: []}                                     # interface -> [rect] (with clearance for tests)
    runs = {1: [], 3: []}                                       # interface -> [[rects of one run]]
    vias, port_vias, ends = [], [], []
    via_budget = n_vias

    def free(k, r):
        x0, y0, x1, y1 = r
        return all(x1 + clearance <= a0 or a1 + clearance <= x0 or y1 + clearance <= b0 or b1 + clearance <= y0
                   for a0, b0, a1, b1 in placed[k])

    def seg_rect(p, q, w):
        return (min(p[0], q[0]) - w / 2, min(p[1], q[1]) - w / 2, max(p[0], q[0]) + w / 2, max(p[1], q[1]) + w / 2)

    t = 0
    tries = 0
    while t < n_traces and tries < 20000:
        tries += 1
        w = rng.uniform(*width)
        nseg = int(rng.integers(segments[0], segments[1] + 1))
        k = int(rng.choice([1, 3]))
        p = np.array([rng.uniform(2e-3, W - 2e-3), rng.uniform(2e-3, H - 2e-3)])
        horiz = bool(rng.integers(2))
        pts, layers_ = [p], []
        ok = True
        for s in range(nseg):
            L = rng.uniform(*seg_len) * rng.choice([-1, 1])
            q = pts[-1] + (np.array([L, 0.0]) if horiz else np.array([0.0, L]))
            if not (1e-3 <= q[0] <= W - 1e-3 and 1e-3 <= q[1] <= H - 1e-3):
                ok = False
                break
            pts.append(q)
            horiz = not horiz
        if not ok:
            continue
        # where the trace changes interface: at an inner segment end, while the via budget lasts
        switch = set()
        if via_budget > 0 and nseg >= 2:
            j = int(rng.integers(1, nseg))
            switch.add(j)
        seg_layer, kk = [], k
        for s in range(nseg):
            if s in switch:
                kk = 4 - kk                                     # 1 <-> 3
            seg_layer.append(kk)
        rects = [(seg_layer[s], seg_rect(pts[s], pts[s + 1], w)) for s in range(nseg)]
        # clearance on each interface, including to the other runs of this trace on that interface
        if not all(free(kl, r) for kl, r in rects):
            continue
        is_port_trace = len(port_vias) < n_ports
        # a port via runs from the ground through the lower interfaces: none may have copper on its axis
        if is_port_trace:
            bad = False
            for e, kl in ((pts[0], seg_layer[0]), (pts[-1], seg_layer[-1])):
                for kb in range(1, kl):
                    if kb in placed and _on_copper([r for r in placed[kb]], e[0], e[1], clearance):
                        bad = True
            if bad:
                continue
        for kl, r in rects:
            placed[kl].append(r)
        # runs: consecutive segments on one interface
        cur, cur_k = [], seg_layer[0]
        for s in range(nseg):
            if seg_layer[s] != cur_k:
                runs[cur_k].append(cur)
                cur, cur_k = [], seg_layer[s]
            cur.append(rects[s][1])
        runs[cur_k].append(cur)
        for j in sorted(switch):
            vias.append(Via(pts[j][0], pts[j][1], 1, 3, 0.15e-3, f"V{len(vias) + 1}"))
            via_budget -= 1
        if is_port_trace:
            for e, kl in ((pts[0], seg_layer[0]), (pts[-1], seg_layer[-1])):
                port_vias.append(Via(e[0], e[1], 0, kl, 0.15e-3, f"P{len(port_vias) + 1}"))
        ends.append(pts)
        t += 1
    if t < n_traces:
        raise RuntimeError(f"routed_board: placed {t} of {n_traces} traces")
    # port vias sit at the trace ends: pull them inside the end square so the vertex is on the copper
    all_vias = port_vias + vias
    shapes = {k: [r for run in runs[k] for r in run] for k in (1, 3) if runs[k]}
    nodes, tris, tl = mesh_layers(st, shapes, dmax, ncross=ncross, vias=all_vias,
                                  pieces={k: runs[k] for k in shapes})
    return Board(st, nodes, tris, tl, all_vias, [ViaPort(v, 50.0, v.name) for v in port_vias], dmax, 5.0,
                 f"routed_board(seed={seed})", shapes)
