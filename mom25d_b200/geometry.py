"""
mom25d_b200.geometry - once-per-mesh set-up of the hot path: the packed edge / triangle arrays the fill kernels
read, the quadrature points, via chains and fans, the Green-table interface pairs, and port excitations.

The packing is the reference's (FastOperator.__init__, mom25d fast.py:364-406; Simulation.__init__, sim.py:395-583
for chains, fans and quadrature), so its compiled core and our kernels read identical numbers:

  g: ep, em (int32 [Ne]) T+ / T-; lt (int32 [Nt]) the triangle's interface as an index into `layers`;
     te (int32 [Nt, 3]) the edges of the halves on each triangle (-1: none); ta (f64 [Nt, 3]) their alpha;
     tv (f64 [Nt, 3, 2]) their free vertex; ap, am (f64 [Ne]) alpha on T+ / T-; vp, vm (f64 [Ne, 2]) free
     vertices; cent (f64 [Nt, 2]); area (f64 [Nt])
  q: nodes (f64 [Nn, 2]), tris (int32 [Nt, 3]), P3 (f64 [Nt, 3, 2]), W3 (f64 [Nt, 3]), P6 (f64 [Nt, 6, 2]),
     W6 (f64 [Nt, 6])  (weights include the triangle's area)
"""
import numpy as np

from .board import RWG, BAR3, BAR6, W3, W6, quad_pts, ViaPort, GapPort, LinePort


class Geometry:
    """Everything about a meshed board that does not depend on frequency."""

    def __init__(self, board, near_fac=None):
        self.board, st = board, board.stack
        self.st = st
        self.rwg = r = RWG(board.nodes, board.tris)
        self.tri_layer = np.asarray(board.tri_layer, np.int64)
        self.layers = sorted(set(self.tri_layer.tolist()))
        self.lidx = {k: i for i, k in enumerate(self.layers)}
        self.Ne, self.Nt = r.Ne, len(r.tris)
        self.dmax, self.near_fac = board.dmax, float(near_fac or board.near_fac)
        self.edge_layer = self.tri_layer[r.tp]
        self.tri_idx = {k: np.nonzero(self.tri_layer == k)[0] for k in self.layers}
        V = r.nodes[r.tris]
        self.tri_size = np.linalg.norm(V - np.roll(V, 1, axis=1), axis=2).max(1)        # sim.py:568
        self.P3, self.W3 = quad_pts(r, BAR3), r.area[:, None] * W3[None, :]              # sim.py:569-570
        self.P6, self.W6 = quad_pts(r, BAR6), r.area[:, None] * W6[None, :]
        self.rho_max = 1.05 * np.hypot(*(r.nodes.max(0) - r.nodes.min(0))) + 1e-4       # sim.py:571-572
        self._pack()
        self._vias()
        self.ports = list(board.ports)
        self.N = self.Ne + self.Nv
        self._port_edges()

    # ---- fast.py:377-406 ------------------------------------------------------------------------------------------
    def _pack(self):
        r, Ne = self.rwg, self.Ne
        self.h_tri = np.concatenate([r.tp, r.tm])
        self.h_alpha = np.concatenate([r.l / (2 * r.area[r.tp]), -r.l / (2 * r.area[r.tm])])
        self.h_v = np.vstack([r.vp, r.vm])
        H = -np.ones((self.Nt, 3), np.int64)
        fill = np.zeros(self.Nt, np.int64)
        for h, t in enumerate(self.h_tri):                 # the halves on each triangle in half order
            H[t, fill[t]] = h
            fill[t] += 1
        self.tri_halves = H
        c = np.ascontiguousarray
        self.g = dict(ep=r.tp.astype(np.int32), em=r.tm.astype(np.int32),
                      lt=np.array([self.lidx[k] for k in self.tri_layer], np.int32),
                      te=np.where(H >= 0, H % Ne, -1).astype(np.int32),
                      ta=np.where(H >= 0, self.h_alpha[H], 0.0),
                      tv=np.where((H >= 0)[..., None], self.h_v[H], 0.0),
                      ap=self.h_alpha[:Ne].copy(), am=self.h_alpha[Ne:].copy(), vp=c(self.h_v[:Ne]),
                      vm=c(self.h_v[Ne:]), cent=c(r.cent), area=r.area.copy())
        self.q = dict(nodes=c(r.nodes), tris=r.tris.astype(np.int32), P3=c(self.P3), W3=c(self.W3),
                      P6=c(self.P6), W6=c(self.W6))
        self.tri_z = np.ascontiguousarray(self.st.z[self.tri_layer], float)

    # ---- sim.py:395-414, 537-560: chains, fans and their divergence ------------------------------------------------
    def _vias(self):
        r, st = self.rwg, self.st
        self.vias = list(self.board.vias)
        self.chains, self.via_attach = [], []
        rects = self.board.rects

        def on(v, k):
            return k in rects and any(x0 - 1e-9 <= v.x <= x1 + 1e-9 and y0 - 1e-9 <= v.y <= y1 + 1e-9
                                      for x0, y0, x1, y1 in rects[k])
        for v in self.vias:
            for k in (v.k_bot, v.k_top):
                if not (st.is_pec(k) or on(v, k)):
                    raise ValueError(f"via {v.name} ends on M{k} where there is no metal")
            att = [v.k_bot] + [k for k in range(v.k_bot + 1, v.k_top) if on(v, k)] + [v.k_top]
            self.via_attach.append([k for k in att if k in self.layers])
            self.chains += [(v, a, b) for a, b in zip(att[:-1], att[1:])]
        via_vertex = {}
        for i, v in enumerate(self.vias):
            for k in self.via_attach[i]:
                idx = np.unique(r.tris[self.tri_idx[k]])
                d = np.hypot(r.nodes[idx, 0] - v.x, r.nodes[idx, 1] - v.y)
                j = int(np.argmin(d))
                if d[j] > 1e-9:
                    raise ValueError(f"via {v.name}: not on the M{k} mesh")
                via_vertex[(i, k)] = int(idx[j])
        self.via_vertex = via_vertex
        self.fan = {key: np.nonzero((r.tris == vid).any(1))[0] for key, vid in via_vertex.items()}
        self.F = np.array(sorted({t for v in self.fan.values() for t in v}), int)
        fpos = {t: j for j, t in enumerate(self.F)}
        self.Nv = len(self.chains)
        self.dF = np.zeros((len(self.F), self.Nv))
        for n, (v, kb, kt) in enumerate(self.chains):
            i = self.vias.index(v)
            for k, div in ((kb, +1.0), (kt, -1.0)):
                if (i, k) in self.fan:
                    ts = self.fan[(i, k)]
                    self.dF[[fpos[t] for t in ts], n] += div / r.area[ts].sum()
        # sim.py:786-814: chain positions, spans, and the via-via pairs grouped by span pair
        ch = self.chains
        self.ch_x = np.array([v.x for v, _, _ in ch], float)
        self.ch_y = np.array([v.y for v, _, _ in ch], float)
        a = np.array([v.a for v, _, _ in ch], float)
        via_id = {}
        vid = np.array([via_id.setdefault(id(v), len(via_id)) for v, _, _ in ch], int)
        span_of = [(kb, kt) for _, kb, kt in ch]
        self.spans = sorted(set(span_of))
        si = np.array([self.spans.index(s) for s in span_of], int)
        self.by_span = {s: np.flatnonzero(si == i) for i, s in enumerate(self.spans)}
        m, n = np.triu_indices(len(ch))
        d = np.where(vid[m] == vid[n], a[m], np.maximum(np.hypot(self.ch_x[m] - self.ch_x[n],
                                                                 self.ch_y[m] - self.ch_y[n]), 0.5 * (a[m] + a[n])))
        key = si[m] * len(self.spans) + si[n]
        order = np.argsort(key, kind='stable')
        self.via_groups = {}
        for gk in np.unique(key):
            sel = order[np.searchsorted(key[order], gk, 'left'):np.searchsorted(key[order], gk, 'right')]
            self.via_groups[(self.spans[gk // len(self.spans)], self.spans[gk % len(self.spans)])] = \
                (m[sel], n[sel], d[sel])
        self.ch_a, self.ch_len = a, np.array([st.z[kt] - st.z[kb] for _, kb, kt in ch], float)

    # ---- sim.py:736-745: the interface pairs and which singular parts their tables take out ------------------------
    def table_pairs(self):
        """[(a, b, cross_sing, image_sing)] for every pair of metal interfaces a <= b (sorted: the tables' order)."""
        out = []
        for i, a in enumerate(self.layers):
            for b in self.layers[i:]:
                xs = a != b and abs(self.st.z[a] - self.st.z[b]) < 3 * self.dmax
                im = a == b and self.st.nearest_discontinuity(a) < 1.5 * self.dmax
                out.append((a, b, bool(xs), bool(im)))
        return out

    def tab_index(self):
        """tab (int32 [L, L]): the table of each interface pair (fast.py:556-560)."""
        keys = [(a, b) for a, b, _, _ in self.table_pairs()]
        tab = np.zeros((len(self.layers),) * 2, np.int32)
        for i, (a, b) in enumerate(keys):
            tab[self.lidx[a], self.lidx[b]] = tab[self.lidx[b], self.lidx[a]] = i
        return tab

    # ---- sim.py:706-726, 988-1007: the ports' edges, excitation and port currents -----------------------------------
    def _port_chain(self, p):
        return next(n for n, (v, _, _) in enumerate(self.chains) if v is p.via)

    def line_edges(self, lp, s=0.0, tol=None):
        """sim.py:695-705: the edges on the transverse line at distance s from lp's centre along its direction,
        within its width, on its interface; with their sign along the direction."""
        r = self.rwg
        tol = tol or 1e-3 * self.dmax
        o = lp.c + lp.d * s
        e0, e1 = r.ends[:, 0] - o, r.ends[:, 1] - o
        on = (np.abs(e0 @ lp.d) < tol) & (np.abs(e1 @ lp.d) < tol) & (self.edge_layer == lp.layer)
        on &= (np.abs(e0 @ lp.t) <= lp.w / 2 + tol) & (np.abs(e1 @ lp.t) <= lp.w / 2 + tol)
        idx = np.nonzero(on)[0]
        return idx, np.sign(r.nrm[idx] @ lp.d)

    def gap_edges(self, p, tol=None):
        """The edges of a gap port's (or a lumped element's, or a wave port's source) transverse line."""
        return self.line_edges(p, 0.0, tol)

    def _port_edges(self):
        """sim.py:706-726: each port's source edges, and a wave port's sample positions and cut edges."""
        self.samples, self.cuts, self.gaps = [], [], []
        for p in self.ports:
            if isinstance(p, ViaPort):
                self.samples.append(None); self.cuts.append(None); self.gaps.append(None)
                continue
            gap = self.gap_edges(p)
            if not len(gap[0]):
                raise ValueError(f"port {p.name}: no mesh edges on the gap line")
            self.gaps.append(gap)
            if isinstance(p, LinePort):
                s = p.sample_positions(self.dmax)
                cuts = [self.line_edges(p, x) for x in s]
                if not all(len(c[0]) for c in cuts):
                    raise ValueError(f"port {p.name}: a sample cut off the conductor")
                self.samples.append(s); self.cuts.append(cuts)
            else:
                self.samples.append(None); self.cuts.append(None)

    def excitation(self):
        E = np.zeros((self.N, len(self.ports)), complex)
        for j, p in enumerate(self.ports):
            if isinstance(p, ViaPort):
                E[self.Ne + self._port_chain(p), j] = p.sign
            else:
                idx, sig = self.gaps[j]
                E[idx, j] = sig * self.rwg.l[idx]
        return E

    def port_rows(self):
        """Every row of I that S needs: the via ports' chains, the gap ports' edges, the wave ports' cut edges."""
        rows = []
        for j, p in enumerate(self.ports):
            if isinstance(p, ViaPort):
                rows.append([self.Ne + self._port_chain(p)])
            elif isinstance(p, LinePort):
                rows += [idx for idx, _ in self.cuts[j]]
            else:
                rows.append(self.gaps[j][0])
        return np.unique(np.concatenate(rows).astype(np.int64)) if rows else np.zeros(0, np.int64)

    def port_currents(self, I):
        """(nports, ncols): each port's current at its source for every excitation column (sim.py:997-1003)."""
        out = np.zeros((len(self.ports), I.shape[1]), complex)
        for j, p in enumerate(self.ports):
            if isinstance(p, ViaPort):
                out[j] = p.sign * I[self.Ne + self._port_chain(p)]
            else:
                idx, sig = self.gaps[j]
                out[j] = ((sig * self.rwg.l[idx])[:, None] * I[idx]).sum(0)
        return out

    def cut_currents(self, I, j):
        """(n_cuts, ncols): the currents through wave port j's sample cuts (sim.py:1005-1007)."""
        l = self.rwg.l
        return np.array([((sig * l[idx])[:, None] * I[idx]).sum(0) for idx, sig in self.cuts[j]])

    def sparams_from_currents(self, I, f=None, info=None):
        """S from the currents of the excitation columns (sim.py:1045-1092): a lumped (via or gap) port's waves
        A = (V + zc I) / (2 sqrt zc), B = (V - zc I) / (2 sqrt zc), V the unit EMF of each column; a wave port's
        from the forward and backward waves fitted on its feed (ports.wave_port_waves); S = B A^-1, made reciprocal
        when there are wave ports (ports.balance). info (a dict), where given, gets gamma, the fit residuals and
        the ports' scales."""
        from .ports import balance, wave_port_waves
        n = len(self.ports)
        Ip = self.port_currents(I)
        Ap, Bp = np.zeros((n, n), complex), np.zeros((n, n), complex)
        gam, resid, low = np.full(n, np.nan + 0j), np.zeros(n), []
        for i, p in enumerate(self.ports):
            if getattr(p, 'zc_fn', None) is not None and f is not None:
                p.zc = float(p.zc_fn(f))
            if isinstance(p, LinePort):
                Ap[i], Bp[i], gam[i], resid[i], span = wave_port_waves(p, self.samples[i], self.cut_currents(I, i), f)
                if span < 0.4:
                    low.append(p.name)
            elif isinstance(p, (ViaPort, GapPort)):
                Vp = np.eye(n)[i]
                Ap[i], Bp[i] = (Vp + p.zc * Ip[i]) / (2 * np.sqrt(p.zc)), (Vp - p.zc * Ip[i]) / (2 * np.sqrt(p.zc))
            else:
                raise NotImplementedError(f"port {getattr(p, 'name', p)}: via, gap or wave (LinePort) ports")
        S = Bp @ np.linalg.inv(Ap)
        wave = np.array([isinstance(p, LinePort) for p in self.ports])
        scale = np.ones(n)
        if wave.any() and n > 1:
            S, scale = balance(S, ~wave)
        if info is not None:
            info.update(gamma=gam, resid=resid, scale=scale, low_span=low)
        return S
