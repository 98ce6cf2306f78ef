// fill.cu - the per-frequency impedance-matrix fill on the GPU: centroid-rule far field, near-field correction,
// near-pair search, via-fan charge moments, radial-table sums, the matrix-free far-field product and the symmetric
// equilibration. Restates mom25d_core.cpp (cited per kernel) with one thread per matrix entry / triangle pair.
#include "common.cuh"

// ---- the tabulated kernel (mom25d_core.cpp:64-90) ---------------------------------------------------------------------
// TB: m25_tables (complex128 samples) or m25_tables_f (complex64); R the arithmetic precision.
template <typename R, typename TB>
__device__ __forceinline__ void tab_rest(const TB &tb, int t, R r, cpx<R> &ga, cpx<R> &gq)
{
    R u = r / (R)tb.dr[t];
    const R umax = (R)tb.nfine - (R)1.000001;
    if (u > umax) u = umax;
    int i = (int)u;
    R f = u - (R)i;
    size_t o = (size_t)t * tb.nfine + i;
    cpx<R> a0 = ldc<R>((const R *)tb.A, o), a1 = ldc<R>((const R *)tb.A, o + 1);
    cpx<R> q0 = ldc<R>((const R *)tb.Q, o), q1 = ldc<R>((const R *)tb.Q, o + 1);
    ga = a0 * (1 - f) + a1 * f;
    gq = q0 * (1 - f) + q1 * f;
}

template <typename R, typename TB>
__device__ __forceinline__ void tab_kern(const TB &tb, int la, int lb, R r, cpx<R> &ga, cpx<R> &gq)
{
    int t = tb.tab[la * tb.L + lb];
    tab_rest<R>(tb, t, r, ga, gq);
    int kd = tb.kind[t];
    if (kd == 0) {
        if (r > 0) {
            ga += ldc<R>((const R *)tb.cA, t) / r;
            gq += ldc<R>((const R *)tb.cq, t) / r;
        }
        R di = (R)tb.dimg[t];
        if (di > 0) {
            R ri = (R)1 / sqrt(r * r + di * di);
            ga += ldc<R>((const R *)tb.cAi, t) * ri;
            gq += ldc<R>((const R *)tb.cqi, t) * ri;
        }
    } else if (kd == 1) {
        R dd = (R)tb.d[t];
        R ri = (R)1 / sqrt(r * r + dd * dd);
        ga += ldc<R>((const R *)tb.cA, t) * ri;
        gq += ldc<R>((const R *)tb.cq, t) * ri;
    }
}

// centroid distance: the differences in double (nearby triangles' coordinates cancel), the root in R
template <typename R>
__device__ __forceinline__ R cdist(const double *c, int p, int q)
{
    double dx = c[2 * p] - c[2 * q], dy = c[2 * p + 1] - c[2 * q + 1];
    return sqrt((R)(dx * dx + dy * dy));
}

// ---- far field: fill_far (mom25d_core.cpp:132-173) ----------------------------------------------------------------
// A 32 x 32 tile of edges per block. The reference evaluates the tabulated kernel 4 times per entry (one per pair
// of the two edges' triangles); here the tile's distinct row and column triangles are found first (about 31 of
// each for 32 edges), the kernel is evaluated once per distinct triangle pair into shared memory, and every entry
// is assembled from four shared-memory lookups (0.95 evaluations an entry instead of 4). Each entry (m, n) is
// formed in the reference's order for the pair (min(m, n), max(m, n)) and the kernel is symmetric in its two
// triangles (distance, symmetric table map), so Z is exactly symmetric, as the reference writes it. A tile whose
// distinct pairs do not fit the shared-memory budget evaluates its entries directly.
struct EdgeHalves { int p[2]; int lt[2]; double a[2], dx[2], dy[2]; };

#define FF_SMEM (48 * 1024)

template <typename R, typename TB>
__device__ __forceinline__ void fill_far_tile(R *Z, long ld, const m25_mesh &g, const TB &tb, double w)
{
    typedef cpx<R> C;
    extern __shared__ __align__(16) unsigned char ff_raw[];
    constexpr int GCAP = FF_SMEM / (2 * sizeof(C));                   // distinct triangle pairs a tile holds
    C *gas = reinterpret_cast<C *>(ff_raw), *gqs = gas + GCAP;
    __shared__ EdgeHalves rows[32], cols[32];
    __shared__ short uid[2][64];                                      // [row / col][edge half 2 e + s] -> distinct index
    __shared__ int tri[2][64];                                        // distinct triangles, in first-seen order
    __shared__ unsigned rep_mask[2][2];
    __shared__ int nu[2];
    const int M0 = blockIdx.y * 32, N0 = blockIdx.x * 32;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    if (tid < 64) {
        int e = (tid < 32 ? M0 : N0) + (tid & 31);
        EdgeHalves h;
        if (e < g.Ne) {
            int pp = g.ep[e], pm = g.em[e];
            h.p[0] = pp; h.p[1] = pm;
            h.lt[0] = g.lt[pp]; h.lt[1] = g.lt[pm];
            h.a[0] = g.ap[e] * g.area[pp]; h.a[1] = g.am[e] * g.area[pm];
            h.dx[0] = g.cent[2 * pp] - g.vp[2 * e]; h.dy[0] = g.cent[2 * pp + 1] - g.vp[2 * e + 1];
            h.dx[1] = g.cent[2 * pm] - g.vm[2 * e]; h.dy[1] = g.cent[2 * pm + 1] - g.vm[2 * e + 1];
        } else {
            h.p[0] = h.p[1] = 0; h.lt[0] = h.lt[1] = 0; h.a[0] = h.a[1] = 0; h.dx[0] = h.dx[1] = h.dy[0] = h.dy[1] = 0;
        }
        (tid < 32 ? rows : cols)[tid & 31] = h;
    }
    __syncthreads();
    // distinct triangles of the row halves (threads 0 .. 63) and of the column halves (64 .. 127): a half is its
    // triangle's representative when no earlier half has the triangle; representatives are numbered by a ballot
    int side = tid >> 6, hh = tid & 63, first = -1, x = -1;
    if (tid < 128) {
        const EdgeHalves *E = side ? cols : rows;
        x = E[hh >> 1].p[hh & 1];
        for (int j = 0; j < hh; ++j)
            if (E[j >> 1].p[j & 1] == x) { first = j; break; }
        const unsigned m = __ballot_sync(0xffffffffu, first < 0);
        if ((tid & 31) == 0) rep_mask[side][(tid >> 5) & 1] = m;
    }
    __syncthreads();
    if (tid < 128 && first < 0) {
        const unsigned lo = rep_mask[side][0], hi = rep_mask[side][1];
        const int id = hh < 32 ? __popc(lo & ((1u << hh) - 1u)) : __popc(lo) + __popc(hi & ((1u << (hh - 32)) - 1u));
        uid[side][hh] = (short)id;
        tri[side][id] = x;
    }
    if (tid < 2) nu[tid] = __popc(rep_mask[tid][0]) + __popc(rep_mask[tid][1]);
    __syncthreads();
    if (tid < 128 && first >= 0) uid[side][hh] = uid[side][first];
    __syncthreads();
    const int nr = nu[0], nc = nu[1];
    const bool tabled = nr * nc <= GCAP;
    if (tabled) {
        for (int q = tid; q < nr * nc; q += 256) {
            const int i = q / nc, j = q - i * nc, p = tri[0][i], t = tri[1][j];
            C ga, gq;
            tab_kern<R>(tb, g.lt[p], g.lt[t], cdist<R>(g.cent, p, t), ga, gq);
            gas[q] = ga;
            gqs[q] = gq;
        }
    }
    __syncthreads();
    const int n = N0 + threadIdx.x;
    if (n >= g.Ne) return;
    const C jw = mk<R>(0, (R)w);
    const C inv_jw = mk<R>(0, (R)(-1.0 / w));
    for (int i = threadIdx.y; i < 32; i += 8) {
        const int m = M0 + i;
        if (m >= g.Ne) break;
        const bool up = m <= n;
        const EdgeHalves &A = up ? rows[i] : cols[threadIdx.x];
        const EdgeHalves &B = up ? cols[threadIdx.x] : rows[i];
        C v = mk<R>(0, 0);
        for (int s = 0; s < 2; ++s)
            for (int t = 0; t < 2; ++t) {
                C ga, gq;
                if (tabled) {
                    // the row-side index of the pair is the row edge's half, whichever of A, B that is
                    const int ir = up ? uid[0][2 * i + s] : uid[0][2 * i + t];
                    const int ic = up ? uid[1][2 * threadIdx.x + t] : uid[1][2 * threadIdx.x + s];
                    ga = gas[ir * nc + ic];
                    gq = gqs[ir * nc + ic];
                } else {
                    tab_kern<R>(tb, A.lt[s], B.lt[t], cdist<R>(g.cent, A.p[s], B.p[t]), ga, gq);
                }
                R dot = (R)A.dx[s] * (R)B.dx[t] + (R)A.dy[s] * (R)B.dy[t];
                C term = (jw * dot) * ga + (gq * (R)4) * inv_jw;
                v += ((R)A.a[s] * (R)B.a[t]) * term;
            }
        stc<R>(Z, (size_t)m * ld + n, v);
    }
}

// four CTAs an SM (64 registers; 88 let two): the tile's phases end in barriers, and the other CTAs' warps fill
// those stalls (routed board, N = 18,788: the FP64 fill phase 15.5 -> 12.3 ms; three CTAs 12.6)
template <typename R, typename TB>
__global__ void __launch_bounds__(256, 4) k_fill_far(R *Z, long ld, m25_mesh g, TB tb, double w)
{
    fill_far_tile<R, TB>(Z, ld, g, tb, w);
}

// Several frequencies of one board in one launch: grid z is the frequency, each with its own Z, tables and w (the
// batched sweep: the far part of every frequency's Z, the tables of all of them resident).
template <typename R, typename TB>
__global__ void __launch_bounds__(256, 4) k_fill_far_multi(R *const *Zs, long ld, m25_mesh g, const TB *tbs,
                                                        const double *ws)
{
    const int f = blockIdx.z;
    const TB tb = tbs[f];
    fill_far_tile<R, TB>(Zs[f], ld, g, tb, ws[f]);
}

// far_block (mom25d_core.cpp:176-211): arbitrary row / column edge lists, complex128 out
template <typename TB>
__global__ void k_far_block(const int *R_, int nr, const int *C_, int nc, double *out, m25_mesh g, TB tb, double w)
{
    long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (idx >= (long)nr * nc) return;
    int i = idx / nc, j = idx % nc;
    int m = R_[i], n = C_[j];
    const zd jw = mk<double>(0, w), inv_jw = mk<double>(0, -1.0 / w);
    int pm[2] = {g.ep[m], g.em[m]}, pn[2] = {g.ep[n], g.em[n]};
    double am_[2] = {g.ap[m] * g.area[pm[0]], g.am[m] * g.area[pm[1]]};
    double dx[2] = {g.cent[2 * pm[0]] - g.vp[2 * m], g.cent[2 * pm[1]] - g.vm[2 * m]};
    double dy[2] = {g.cent[2 * pm[0] + 1] - g.vp[2 * m + 1], g.cent[2 * pm[1] + 1] - g.vm[2 * m + 1]};
    double an[2] = {g.ap[n] * g.area[pn[0]], g.am[n] * g.area[pn[1]]};
    double ex[2] = {g.cent[2 * pn[0]] - g.vp[2 * n], g.cent[2 * pn[1]] - g.vm[2 * n]};
    double ey[2] = {g.cent[2 * pn[0] + 1] - g.vp[2 * n + 1], g.cent[2 * pn[1] + 1] - g.vm[2 * n + 1]};
    zd v = mk<double>(0, 0);
    for (int s = 0; s < 2; ++s)
        for (int t = 0; t < 2; ++t) {
            zd ga, gq;
            tab_kern<double>(tb, g.lt[pm[s]], g.lt[pn[t]], cdist<double>(g.cent, pm[s], pn[t]), ga, gq);
            zd term = (jw * (dx[s] * ex[t] + dy[s] * ey[t])) * ga + (gq * 4.0) * inv_jw;
            v += (am_[s] * an[t]) * term;
        }
    stc<double>(out, idx, v);
}

// ---- near-field correction (the reference's near_core, mom25d_core.cpp:417-507): a half warp per near pair ---------
// A near pair (p, q) of triangles gets: the smooth rest of the tabulated kernel integrated by the 3-point (same
// interface) or 6-point (across interfaces) rule on both triangles; plus each extracted singular part c / sqrt(rho^2
// + d^2) integrated analytically over one triangle of the pair with the 6-point rule over the other (the rule goes
// on the smaller triangle, ties by index: mom25d_core.cpp:321-324); minus the centroid value the far fill put there.
// What is integrated are seven moments: 1, r, r', r.r' against G_A and 1 against G_q (r on p, r' on q); the 3 x 3
// values of the edge pairs (halves on p) x (halves on q) are combinations of them.
//
// On the GPU, 16 lanes (a half warp) carry one pair, two pairs a warp:
//  1. the np^2 quadrature point pairs (9 or 36) are dealt out over the 16 lanes, each lane sums its share of the
//     seven moments, and a butterfly of shuffles inside the half warp gives every lane the totals;
//  2. the analytic moments (computed at the first frequency only: `stat` keeps them, they do not depend on it) deal
//     out their 18 (rule point, triangle side) line integrals the same way;
//  3. lanes 0 .. 8 each form one of the 3 x 3 edge-pair values and add it into Z (mode 0) or write it as a COO
//     triplet (mode 2, slot 9 i + 3 s + u, row -1 where a half is missing).
// The line integrals of 1/R and of the in-plane offset over a triangle side seen from a point at height d are the
// closed forms of Wilton et al. (IEEE Trans. AP 32, 1984) and Graglia (IEEE Trans. AP 41, 1993).

__device__ __forceinline__ bool rule_on_p(double ap, double aq, int p, int q)
{
    const double tie = 1e-9 * fmax(ap, aq);
    return fabs(ap - aq) <= tie ? p <= q : ap < aq;
}

__device__ __forceinline__ double half_sum(double v, unsigned mask)
{
    v += __shfl_xor_sync(mask, v, 8, 16);
    v += __shfl_xor_sync(mask, v, 4, 16);
    v += __shfl_xor_sync(mask, v, 2, 16);
    v += __shfl_xor_sync(mask, v, 1, 16);
    return v;
}

__device__ __forceinline__ zd half_sum(zd v, unsigned mask) { return mk<double>(half_sum(v.x, mask), half_sum(v.y, mask)); }

// The line integral of side `side` of triangle `tri` (counter-clockwise) seen from the point r at height d:
// this side's part of I1 = int 1/R dS' and of IR = int (r' - r)/R dS' (in-plane) over the triangle.
__device__ __forceinline__ void side_integrals(const m25_quad &q, int tri, int side, double rx, double ry, double d,
                                               double &I1, double &IRx, double &IRy)
{
    const int n0 = q.tris[3 * tri + side], n1 = q.tris[3 * tri + (side == 2 ? 0 : side + 1)];
    const double v0x = q.nodes[2 * n0], v0y = q.nodes[2 * n0 + 1];
    const double ex = q.nodes[2 * n1] - v0x, ey = q.nodes[2 * n1 + 1] - v0y;
    const double len = sqrt(ex * ex + ey * ey);
    const double tx = ex / len, ty = ey / len;             // along the side; (ty, -tx) points out of the triangle
    const double ox = v0x - rx, oy = v0y - ry;
    const double s0 = ox * tx + oy * ty, s1 = s0 + len;    // the side's ends along it, from the foot of r
    const double h = ox * ty - oy * tx;                    // signed in-plane distance of r from the side's line
    const double ad = fabs(d);
    const double rho2 = h * h + d * d, rho = sqrt(rho2);
    const double R0 = sqrt(rho2 + s0 * s0), R1 = sqrt(rho2 + s1 * s1);
    const double lg = rho > 1e-14 * len ? asinh(s1 / rho) - asinh(s0 / rho) : 0.0;
    const double ang = atan2(h * s1, rho2 + ad * R1) - atan2(h * s0, rho2 + ad * R0);
    I1 = h * lg - ad * ang;
    const double e = 0.5 * (rho2 * lg + s1 * R1 - s0 * R0);
    IRx = e * ty;
    IRy = -e * tx;
}

template <typename Zt>
__device__ __forceinline__ void add_to_z(Zt *Z, size_t i, zd v);
template <> __device__ __forceinline__ void add_to_z<double>(double *Z, size_t i, zd v)
{
    atomicAdd(Z + 2 * i, v.x); atomicAdd(Z + 2 * i + 1, v.y);
}
template <> __device__ __forceinline__ void add_to_z<float>(float *Z, size_t i, zd v)
{
    atomicAdd(Z + 2 * i, (float)v.x); atomicAdd(Z + 2 * i + 1, (float)v.y);
}

template <typename Zt>
__global__ void __launch_bounds__(256) k_near(int mode, Zt *Z, long ld, int *ri, int *ci, double *vv, double *qcorr,
                                              double *stat, int stat_ready, m25_mesh g, m25_tables tb, m25_quad q,
                                              const int *P, const int *Q, long n, double w, int *err)
{
    const long i = (blockIdx.x * (long)blockDim.x + threadIdx.x) >> 4;     // the pair of this half warp
    if (i >= n) return;                                                   // (whole half warps leave together)
    const int l = threadIdx.x & 15;
    const unsigned mask = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
    const int p = P[i], qq = Q[i];
    if (p < 0 || p >= g.Nt || qq < 0 || qq >= g.Nt) {
        if (l == 0) dev_error(err, M25_DEV_INDEX);
        return;
    }
    const int la = g.lt[p], lb = g.lt[qq];
    const int t = tb.tab[la * tb.L + lb];
    const int np = la == lb ? 3 : 6;
    const double *Pa = np == 3 ? q.P3 + 6 * (size_t)p : q.P6 + 12 * (size_t)p;
    const double *Pb = np == 3 ? q.P3 + 6 * (size_t)qq : q.P6 + 12 * (size_t)qq;
    const double *Wa = np == 3 ? q.W3 + 3 * (size_t)p : q.W6 + 6 * (size_t)p;
    const double *Wb = np == 3 ? q.W3 + 3 * (size_t)qq : q.W6 + 6 * (size_t)qq;
    // 1. the smooth rest by quadrature: moments 1, r (obs), r' (src), r.r' of G_A and 1 of G_q
    zd s1 = mk<double>(0, 0), sox = s1, soy = s1, ssx = s1, ssy = s1, srr = s1, sq = s1;
    for (int k = l; k < np * np; k += 16) {
        const int a = k / np, b = k - a * np;
        const double ax = Pa[2 * a], ay = Pa[2 * a + 1], bx = Pb[2 * b], by = Pb[2 * b + 1];
        const double dx = ax - bx, dy = ay - by;
        zd ga, gq;
        tab_rest<double>(tb, t, sqrt(dx * dx + dy * dy), ga, gq);
        const double wt = Wa[a] * Wb[b];
        ga = ga * wt;
        s1 += ga; sox += ga * ax; soy += ga * ay; ssx += ga * bx; ssy += ga * by;
        srr += ga * (ax * bx + ay * by);
        sq += gq * wt;
    }
    s1 = half_sum(s1, mask); sox = half_sum(sox, mask); soy = half_sum(soy, mask);
    ssx = half_sum(ssx, mask); ssy = half_sum(ssy, mask); srr = half_sum(srr, mask); sq = half_sum(sq, mask);
    // 2. the extracted singular parts: the rule on the smaller triangle, the closed form over the other
    const bool obs_rule = rule_on_p(g.area[p], g.area[qq], p, qq);
    const int tr = obs_rule ? p : qq, ta = obs_rule ? qq : p;
    const int kd = tb.kind[t];
    const int nsing = kd == 0 ? (tb.dimg[t] > 0 ? 2 : 1) : (kd == 1 ? 1 : 0);
    for (int x = 0; x < nsing; ++x) {
        const double d = kd == 0 ? (x == 0 ? 0.0 : tb.dimg[t]) : tb.d[t];
        double m[6];                                       // 1, r (obs) x/y, r' (src) x/y, r.r'
        double *kept = stat ? stat + 12 * (size_t)i + 6 * x : nullptr;
        if (kept && stat_ready) {
            for (int c = 0; c < 6; ++c) m[c] = kept[c];
        } else {
            double c0 = 0, crx = 0, cry = 0, cax = 0, cay = 0, crr = 0;    // rule-side r, analytic-side r'
            for (int e = l; e < 18; e += 16) {
                const int kq = e / 3, side = e - 3 * kq;
                const double rx = q.P6[12 * (size_t)tr + 2 * kq], ry = q.P6[12 * (size_t)tr + 2 * kq + 1];
                const double wq = q.W6[6 * (size_t)tr + kq];
                double I1, IRx, IRy;
                side_integrals(q, ta, side, rx, ry, d, I1, IRx, IRy);
                const double Ax = IRx + rx * I1, Ay = IRy + ry * I1;       // int r'/R
                c0 += wq * I1;
                crx += wq * rx * I1; cry += wq * ry * I1;
                cax += wq * Ax; cay += wq * Ay;
                crr += wq * (rx * Ax + ry * Ay);
            }
            m[0] = half_sum(c0, mask);
            const double rx_ = half_sum(crx, mask), ry_ = half_sum(cry, mask);
            const double ax_ = half_sum(cax, mask), ay_ = half_sum(cay, mask);
            m[5] = half_sum(crr, mask);
            if (obs_rule) { m[1] = rx_; m[2] = ry_; m[3] = ax_; m[4] = ay_; }
            else { m[1] = ax_; m[2] = ay_; m[3] = rx_; m[4] = ry_; }
            if (kept && l == 0)
                for (int c = 0; c < 6; ++c) kept[c] = m[c];
        }
        const zd cA = x == 0 ? ldc<double>(tb.cA, t) : ldc<double>(tb.cAi, t);
        const zd cq = x == 0 ? ldc<double>(tb.cq, t) : ldc<double>(tb.cqi, t);
        s1 += cA * m[0]; sox += cA * m[1]; soy += cA * m[2]; ssx += cA * m[3]; ssy += cA * m[4]; srr += cA * m[5];
        sq += cq * m[0];
    }
    // minus the centroid-rule value of the far fill
    {
        zd ga, gq;
        tab_kern<double>(tb, la, lb, cdist<double>(g.cent, p, qq), ga, gq);
        const double wt = g.area[p] * g.area[qq];
        const double ox = g.cent[2 * p], oy = g.cent[2 * p + 1], sx = g.cent[2 * qq], sy = g.cent[2 * qq + 1];
        ga = ga * wt;
        s1 -= ga; sox -= ga * ox; soy -= ga * oy; ssx -= ga * sx; ssy -= ga * sy; srr -= ga * (ox * sx + oy * sy);
        sq -= gq * wt;
    }
    if (qcorr && l == 0) stc<double>(qcorr, i, sq);
    // 3. one edge pair a lane
    if (l >= 9) return;
    const int s = l / 3, u = l - 3 * (l / 3);
    const int em_ = g.te[3 * p + s], en = g.te[3 * qq + u];
    const size_t slot = 9 * (size_t)i + l;
    if (em_ < 0 || en < 0) {
        if (mode == 2) { ri[slot] = -1; ci[slot] = 0; vv[2 * slot] = 0; vv[2 * slot + 1] = 0; }
        return;
    }
    const double am = g.ta[3 * p + s], vx = g.tv[6 * p + 2 * s], vy = g.tv[6 * p + 2 * s + 1];
    const double an = g.ta[3 * qq + u], wx = g.tv[6 * qq + 2 * u], wy = g.tv[6 * qq + 2 * u + 1];
    // int (r - v).(r' - w) G_A and int G_q, from the moments
    const zd vecA = srr - (sox * wx + soy * wy) - (ssx * vx + ssy * vy) + s1 * (vx * wx + vy * wy);
    const zd val = (am * an) * (mk<double>(0, w) * vecA + (sq * 4.0) * mk<double>(0, -1.0 / w));
    if (mode == 0) add_to_z<Zt>(Z, (size_t)em_ * ld + en, val);
    else { ri[slot] = em_; ci[slot] = en; stc<double>(vv, slot, val); }
}

// ---- near pairs (mom25d_core.cpp:1216-1263): brute force over all pairs, rows in order -------------------------------
__global__ void k_near_count(const double *c, const double *sz, const double *zz, int Nt, double fac, long long *cnt)
{
    // one warp per row p
    int p = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
    if (p >= Nt) return;
    double cx = c[2 * p], cy = c[2 * p + 1], zp = zz[p], sp = sz[p];
    long long k = 0;
    for (int q = lane; q < Nt; q += 32) {
        double dx = cx - c[2 * q], dy = cy - c[2 * q + 1], dz = zp - zz[q];
        double R = fac * fmax(sp, sz[q]);
        k += (dx * dx + dy * dy + dz * dz < R * R);
    }
    for (int o = 16; o; o >>= 1) k += __shfl_xor_sync(0xffffffffu, k, o);
    if (lane == 0) cnt[p] = k;
}

__global__ void k_near_fill(const double *c, const double *sz, const double *zz, int Nt, double fac,
                            const long long *off, int *P, int *Q)
{
    int p = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
    if (p >= Nt) return;
    double cx = c[2 * p], cy = c[2 * p + 1], zp = zz[p], sp = sz[p];
    long long base = off[p];
    for (int q0 = 0; q0 < Nt; q0 += 32) {
        int q = q0 + lane;
        bool hit = false;
        if (q < Nt) {
            double dx = cx - c[2 * q], dy = cy - c[2 * q + 1], dz = zp - zz[q];
            double R = fac * fmax(sp, sz[q]);
            hit = dx * dx + dy * dy + dz * dz < R * R;
        }
        unsigned msk = __ballot_sync(0xffffffffu, hit);
        if (hit) {
            long long k = base + __popc(msk & ((1u << lane) - 1));
            P[k] = p; Q[k] = q;
        }
        base += __popc(msk);
    }
}

__global__ void k_exclusive_scan_small(long long *a, int n, long long *total)
{
    // single block, serial chunks: n is the triangle count (<= a few 1e5)
    __shared__ long long part[1024];
    int t = threadIdx.x, nt = blockDim.x;
    int chunk = (n + nt - 1) / nt, b = t * chunk, e = min(n, b + chunk);
    long long s = 0;
    for (int i = b; i < e; ++i) s += a[i];
    part[t] = s;
    __syncthreads();
    if (t == 0) {
        long long acc = 0;
        for (int i = 0; i < nt; ++i) { long long v = part[i]; part[i] = acc; acc += v; }
        *total = acc;
    }
    __syncthreads();
    long long acc = part[t];
    for (int i = b; i < e; ++i) { long long v = a[i]; a[i] = acc; acc += v; }
    if (t == nt - 1) a[n] = *total;
}

// ---- fan charges (fan_q, mom25d_core.cpp:1585-1603) -----------------------------------------------------------------
__global__ void k_fan_q(const int *F, int nf, double *out, m25_mesh g, m25_tables tb)
{
    long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (idx >= (long)g.Nt * nf) return;
    int t = idx / nf, j = idx % nf, f = F[j];
    zd ga, gq;
    tab_kern<double>(tb, g.lt[t], g.lt[f], cdist<double>(g.cent, t, f), ga, gq);
    stc<double>(out, idx, gq * (g.area[t] * g.area[f]));
}

// ---- radial table sums (radial_table_sum, mom25d_core.cpp:1269-1298) ------------------------------------------------
__global__ void k_radial_table_sum(const double *x, const double *y, const double *W, long nt, int nq,
                                   const double *ax, const double *ay, int nv, const double *D, long n, double dr,
                                   double *out)
{
    long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (idx >= nt * nv) return;
    long t = idx / nv;
    int v = idx % nv;
    const double top = (double)n - 1.000001;
    zd acc = mk<double>(0, 0);
    for (int q = 0; q < nq; ++q) {
        const double rx = x[t * nq + q] - ax[v], ry = y[t * nq + q] - ay[v];
        double u = fmin(hypot(rx, ry) / dr, top);
        long i = (long)u;
        double f = u - (double)i;
        acc += (ldc<double>(D, i) * (1.0 - f) + ldc<double>(D, i + 1) * f) * W[t * nq + q];
    }
    stc<double>(out, idx, acc);
}

// ---- matrix-free far product (matvec_far_multi, mom25d_core.cpp:257-314) --------------------------------------------
// 1. per triangle: s0 = sum a A x, s1 = sum a A x (c - v) over the halves on it (gathered through te / ta / tv)
__global__ void k_mv_aggregate(const double *X, int K, m25_mesh g, double *s0, double *s1x, double *s1y)
{
    long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (idx >= (long)g.Nt * K) return;
    int t = idx / K, c = idx % K;
    zd a0 = mk<double>(0, 0), ax = a0, ay = a0;
    for (int s = 0; s < 3; ++s) {
        int e = g.te[3 * t + s];
        if (e < 0) continue;
        zd x = ldc<double>(X, (size_t)e * K + c);
        zd a = x * (g.ta[3 * t + s] * g.area[t]);
        a0 += a;
        ax += a * (g.cent[2 * t] - g.tv[6 * t + 2 * s]);
        ay += a * (g.cent[2 * t + 1] - g.tv[6 * t + 2 * s + 1]);
    }
    stc<double>(s0, idx, a0); stc<double>(s1x, idx, ax); stc<double>(s1y, idx, ay);
}

// 2. vAx[p] = sum_q GA(p, q) s1x[q], vAy likewise, wQ[p] = sum_q GQ(p, q) s0[q]: a block of 128 observation
//    triangles per CTA, source triangles streamed through shared memory; K <= 16 columns.
template <int KMAX>
__global__ void __launch_bounds__(128) k_mv_pairs(int K, m25_mesh g, m25_tables tb, const double *s0,
                                                  const double *s1x, const double *s1y, double *vAx, double *vAy,
                                                  double *wQ)
{
    constexpr int QT = KMAX <= 8 ? 64 : 32;            // source triangles a stage (48 KB of static shared memory)
    __shared__ double sc[QT][2];
    __shared__ int sl[QT];
    __shared__ zd S0[QT][KMAX], SX[QT][KMAX], SY[QT][KMAX];
    const int p = blockIdx.x * 128 + threadIdx.x;
    const bool live = p < g.Nt;
    const double cx = live ? g.cent[2 * p] : 0, cy = live ? g.cent[2 * p + 1] : 0;
    const int lp = live ? g.lt[p] : 0;
    zd ax[KMAX], ay[KMAX], aq[KMAX];
    for (int c = 0; c < KMAX; ++c) ax[c] = ay[c] = aq[c] = mk<double>(0, 0);
    // this block's chunk of source triangles (grid.y chunks; partial sums added atomically)
    const int chunk = (g.Nt + gridDim.y - 1) / gridDim.y;
    const int qb = blockIdx.y * chunk, qe = min(g.Nt, qb + chunk);
    for (int q0 = qb; q0 < qe; q0 += QT) {
        __syncthreads();
        for (int j = threadIdx.x; j < QT; j += 128) {
            int q = q0 + j;
            sc[j][0] = q < qe ? g.cent[2 * q] : 0; sc[j][1] = q < qe ? g.cent[2 * q + 1] : 0;
            sl[j] = q < qe ? g.lt[q] : 0;
        }
        for (int j = threadIdx.x; j < QT * K; j += 128) {
            int qq = j / K, c = j % K, q = q0 + qq;
            zd z0 = mk<double>(0, 0);
            S0[qq][c] = q < qe ? ldc<double>(s0, (size_t)q * K + c) : z0;
            SX[qq][c] = q < qe ? ldc<double>(s1x, (size_t)q * K + c) : z0;
            SY[qq][c] = q < qe ? ldc<double>(s1y, (size_t)q * K + c) : z0;
        }
        __syncthreads();
        if (!live) continue;
        int qn = min(QT, qe - q0);
        for (int j = 0; j < qn; ++j) {
            double dx = cx - sc[j][0], dy = cy - sc[j][1];
            zd ga, gq;
            tab_kern<double>(tb, lp, sl[j], sqrt(dx * dx + dy * dy), ga, gq);
#pragma unroll
            for (int c = 0; c < KMAX; ++c) {
                if (c < K) { ax[c] += ga * SX[j][c]; ay[c] += ga * SY[j][c]; aq[c] += gq * S0[j][c]; }
            }
        }
    }
    if (!live) return;
    for (int c = 0; c < K; ++c) {
        size_t o = 2 * ((size_t)p * K + c);
        atomicAdd(vAx + o, ax[c].x); atomicAdd(vAx + o + 1, ax[c].y);
        atomicAdd(vAy + o, ay[c].x); atomicAdd(vAy + o + 1, ay[c].y);
        atomicAdd(wQ + o, aq[c].x); atomicAdd(wQ + o + 1, aq[c].y);
    }
}

// 3. Y[e] from the two halves' triangle sums
__global__ void k_mv_finish(int K, m25_mesh g, double w, const double *vAx, const double *vAy, const double *wQ,
                            double *Y)
{
    long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (idx >= (long)g.Ne * K) return;
    int e = idx / K, c = idx % K;
    const zd jw = mk<double>(0, w), inv_jw = mk<double>(0, -1.0 / w);
    int p = g.ep[e], q = g.em[e];
    double dpx = g.cent[2 * p] - g.vp[2 * e], dpy = g.cent[2 * p + 1] - g.vp[2 * e + 1];
    double dqx = g.cent[2 * q] - g.vm[2 * e], dqy = g.cent[2 * q + 1] - g.vm[2 * e + 1];
    size_t ip = (size_t)p * K + c, iq = (size_t)q * K + c;
    zd yp = (jw * (ldc<double>(vAx, ip) * dpx + ldc<double>(vAy, ip) * dpy) + (ldc<double>(wQ, ip) * 4.0) * inv_jw)
            * (g.ap[e] * g.area[p]);
    zd ym = (jw * (ldc<double>(vAx, iq) * dqx + ldc<double>(vAy, iq) * dqy) + (ldc<double>(wQ, iq) * 4.0) * inv_jw)
            * (g.am[e] * g.area[q]);
    stc<double>(Y, idx, yp + ym);
}

// ---- equilibration (fast.py:294-305; scale_c64, mom25d_core.cpp:1563-1580) ------------------------------------------
__global__ void k_diag_scale(const double *Z, long n, long ld, double *d)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    zd z = ldc<double>(Z, (size_t)i * ld + i);
    d[i] = 1.0 / sqrt(hypot(z.x, z.y) + 1e-300);
}

__global__ void k_diag_scale_c64(const float *Z, long n, long ld, double *d)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    zf z = ldc<float>(Z, (size_t)i * ld + i);
    d[i] = 1.0 / sqrt(hypot((double)z.x, (double)z.y) + 1e-300);
}

__global__ void k_equilibrate_c64(float *Z, long n, long ld, const double *d)
{
    long i = blockIdx.y;
    double di = d[i];
    for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n; j += (long)gridDim.x * blockDim.x) {
        zf z = ldc<float>(Z, (size_t)i * ld + j);
        float s = (float)(di * d[j]);
        stc<float>(Z, (size_t)i * ld + j, mk<float>(z.x * s, z.y * s));
    }
}

__global__ void k_equilibrate(double *Z, long n, long ld, const double *d, float *Z64)
{
    long i = blockIdx.y;
    double di = d[i];
    for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n; j += (long)gridDim.x * blockDim.x) {
        zd z = ldc<double>(Z, (size_t)i * ld + j) * (di * d[j]);
        stc<double>(Z, (size_t)i * ld + j, z);
        if (Z64) stc<float>(Z64, (size_t)i * n + j, mk<float>((float)z.x, (float)z.y));
    }
}

// ======================================================================================================================
// C ABI
// ======================================================================================================================
static inline cudaStream_t S(void *s) { return (cudaStream_t)s; }
int *m25_dev_err_word();
int m25_check_dev_err(cudaStream_t s, const char *what);

extern "C" int m25_fill_far(void *d_Z, long ld, int single, const m25_mesh *g, const m25_tables *tb,
                            const m25_tables_f *tbf, double w, void *stream)
{
    M25_REQUIRE(d_Z && g && ld >= g->Ne, "m25_fill_far: Z, g and ld >= Ne required");
    if (g->Ne == 0) return M25_OK;
    dim3 grid((g->Ne + 31) / 32, (g->Ne + 31) / 32), block(32, 8);
    if (single) {
        M25_REQUIRE(tbf, "m25_fill_far: single precision needs the complex64 tables");
        M25_CHECK(cudaFuncSetAttribute(k_fill_far<float, m25_tables_f>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       FF_SMEM));
        k_fill_far<float, m25_tables_f><<<grid, block, FF_SMEM, S(stream)>>>((float *)d_Z, ld, *g, *tbf, w);
    } else {
        M25_REQUIRE(tb, "m25_fill_far: the complex128 tables are required");
        M25_CHECK(cudaFuncSetAttribute(k_fill_far<double, m25_tables>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       FF_SMEM));
        k_fill_far<double, m25_tables><<<grid, block, FF_SMEM, S(stream)>>>((double *)d_Z, ld, *g, *tb, w);
    }
    M25_LAUNCH_CHECK("k_fill_far");
    return M25_OK;
}

extern "C" int m25_fill_far_multi(void *const *d_Zs, long ld, int single, const m25_mesh *g, const void *d_tables,
                                  const double *d_w, int nf, void *stream)
{
    M25_REQUIRE(d_Zs && g && d_tables && d_w && ld >= g->Ne && nf >= 1 && nf <= 65535,
                "m25_fill_far_multi: Zs, g, tables, w, ld >= Ne, 1 <= nf <= 65535");
    if (g->Ne == 0) return M25_OK;
    dim3 grid((g->Ne + 31) / 32, (g->Ne + 31) / 32, nf), block(32, 8);
    if (single) {
        M25_CHECK(cudaFuncSetAttribute(k_fill_far_multi<float, m25_tables_f>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, FF_SMEM));
        k_fill_far_multi<float, m25_tables_f><<<grid, block, FF_SMEM, S(stream)>>>(
            (float *const *)d_Zs, ld, *g, (const m25_tables_f *)d_tables, d_w);
    } else {
        M25_CHECK(cudaFuncSetAttribute(k_fill_far_multi<double, m25_tables>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, FF_SMEM));
        k_fill_far_multi<double, m25_tables><<<grid, block, FF_SMEM, S(stream)>>>(
            (double *const *)d_Zs, ld, *g, (const m25_tables *)d_tables, d_w);
    }
    M25_LAUNCH_CHECK("k_fill_far_multi");
    return M25_OK;
}

extern "C" int m25_far_block(const int *d_rows, int nr, const int *d_cols, int nc, double *d_out, const m25_mesh *g,
                             const m25_tables *tb, double w, void *stream)
{
    M25_REQUIRE(g && tb && d_out, "m25_far_block: null argument");
    long tot = (long)nr * nc;
    if (!tot) return M25_OK;
    k_far_block<m25_tables><<<(tot + 255) / 256, 256, 0, S(stream)>>>(d_rows, nr, d_cols, nc, d_out, *g, *tb, w);
    M25_LAUNCH_CHECK("k_far_block");
    return M25_OK;
}

extern "C" int m25_near(int mode, void *d_Z, long ld, int single, int *d_ri, int *d_ci, double *d_vv, double *d_qcorr,
                        double *d_stat, int stat_ready, const m25_mesh *g, const m25_tables *tb, const m25_quad *q,
                        const int *d_P, const int *d_Q, long n, double w, void *stream)
{
    M25_REQUIRE(g && tb && q, "m25_near: null argument");
    M25_REQUIRE(mode == 0 || mode == 2, "m25_near: mode 0 (dense) or 2 (COO)");
    M25_REQUIRE(mode != 0 || (d_Z && ld >= g->Ne), "m25_near: mode 0 needs Z");
    M25_REQUIRE(mode != 2 || (d_ri && d_ci && d_vv), "m25_near: mode 2 needs ri, ci, vv");
    if (n == 0) return M25_OK;
    int *err = m25_dev_err_word();
    const long blocks = (16 * n + 255) / 256;             // 16 lanes a pair
    if (single)
        k_near<float><<<blocks, 256, 0, S(stream)>>>(mode, (float *)d_Z, ld, d_ri, d_ci, d_vv, d_qcorr, d_stat,
                                                     stat_ready, *g, *tb, *q, d_P, d_Q, n, w, err);
    else
        k_near<double><<<blocks, 256, 0, S(stream)>>>(mode, (double *)d_Z, ld, d_ri, d_ci, d_vv, d_qcorr, d_stat,
                                                      stat_ready, *g, *tb, *q, d_P, d_Q, n, w, err);
    M25_LAUNCH_CHECK("k_near");
    return M25_OK;
}

extern "C" int m25_near_pairs(const double *d_cent, const double *d_size, const double *d_z, int Nt, double fac,
                              long long *d_offsets, long long *h_total, int *d_P, int *d_Q, void *stream)
{
    M25_REQUIRE(d_cent && d_size && d_z && d_offsets && h_total, "m25_near_pairs: null argument");
    int blocks = (Nt + 7) / 8;
    if (!d_P) {
        long long *d_tot = d_offsets + Nt;
        k_near_count<<<blocks, 256, 0, S(stream)>>>(d_cent, d_size, d_z, Nt, fac, d_offsets);
        M25_LAUNCH_CHECK("k_near_count");
        k_exclusive_scan_small<<<1, 1024, 0, S(stream)>>>(d_offsets, Nt, d_tot);
        M25_LAUNCH_CHECK("k_exclusive_scan_small");
        M25_CHECK(cudaMemcpyAsync(h_total, d_tot, sizeof(long long), cudaMemcpyDeviceToHost, S(stream)));
        M25_CHECK(cudaStreamSynchronize(S(stream)));
        return M25_OK;
    }
    k_near_fill<<<blocks, 256, 0, S(stream)>>>(d_cent, d_size, d_z, Nt, fac, d_offsets, d_P, d_Q);
    M25_LAUNCH_CHECK("k_near_fill");
    M25_CHECK(cudaStreamSynchronize(S(stream)));
    return M25_OK;
}

extern "C" int m25_fan_q(const int *d_F, int nf, double *d_out, const m25_mesh *g, const m25_tables *tb, void *stream)
{
    M25_REQUIRE(g && tb, "m25_fan_q: null argument");
    long tot = (long)g->Nt * nf;
    if (!tot) return M25_OK;
    k_fan_q<<<(tot + 255) / 256, 256, 0, S(stream)>>>(d_F, nf, d_out, *g, *tb);
    M25_LAUNCH_CHECK("k_fan_q");
    return M25_OK;
}

extern "C" int m25_radial_table_sum(const double *d_px, const double *d_py, const double *d_W, long nt, int nq,
                                    const double *d_vx, const double *d_vy, int nv, const double *d_table, long n,
                                    double dr, double *d_out, void *stream)
{
    M25_REQUIRE(n >= 2 && dr > 0, "m25_radial_table_sum: a table of two points or more, dr > 0");
    long tot = nt * nv;
    if (!tot) return M25_OK;
    k_radial_table_sum<<<(tot + 255) / 256, 256, 0, S(stream)>>>(d_px, d_py, d_W, nt, nq, d_vx, d_vy, nv, d_table,
                                                                  n, dr, d_out);
    M25_LAUNCH_CHECK("k_radial_table_sum");
    return M25_OK;
}

extern "C" int m25_matvec_far_multi(const double *d_X, int K, double *d_Y, double *d_work, const m25_mesh *g,
                                    const m25_tables *tb, double w, void *stream)
{
    M25_REQUIRE(g && tb && d_X && d_Y && d_work, "m25_matvec_far_multi: null argument");
    M25_REQUIRE(K >= 1 && K <= 16, "m25_matvec_far_multi: 1 <= K <= 16 columns a call");
    size_t nk = (size_t)g->Nt * K * 2;
    double *s0 = d_work, *s1x = s0 + nk, *s1y = s1x + nk, *vAx = s1y + nk, *vAy = vAx + nk, *wQ = vAy + nk;
    long tot = (long)g->Nt * K;
    k_mv_aggregate<<<(tot + 255) / 256, 256, 0, S(stream)>>>(d_X, K, *g, s0, s1x, s1y);
    M25_LAUNCH_CHECK("k_mv_aggregate");
    M25_CHECK(cudaMemsetAsync(vAx, 0, 3 * nk * sizeof(double), S(stream)));     // vAx, vAy, wQ: atomic sums
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    dim3 blocks((g->Nt + 127) / 128, 1);
    blocks.y = std::max(1, std::min(64, (4 * sms + (int)blocks.x - 1) / (int)blocks.x));   // ~4 blocks an SM
    if (K <= 4)
        k_mv_pairs<4><<<blocks, 128, 0, S(stream)>>>(K, *g, *tb, s0, s1x, s1y, vAx, vAy, wQ);
    else if (K <= 8)
        k_mv_pairs<8><<<blocks, 128, 0, S(stream)>>>(K, *g, *tb, s0, s1x, s1y, vAx, vAy, wQ);
    else
        k_mv_pairs<16><<<blocks, 128, 0, S(stream)>>>(K, *g, *tb, s0, s1x, s1y, vAx, vAy, wQ);
    M25_LAUNCH_CHECK("k_mv_pairs");
    tot = (long)g->Ne * K;
    k_mv_finish<<<(tot + 255) / 256, 256, 0, S(stream)>>>(K, *g, w, vAx, vAy, wQ, d_Y);
    M25_LAUNCH_CHECK("k_mv_finish");
    return M25_OK;
}

extern "C" int m25_equilibrate(double *d_Z, long n, long ld, const double *d_d, double *d_dsc_out, float *d_Z64,
                               void *stream)
{
    M25_REQUIRE(d_Z && ld >= n, "m25_equilibrate: Z and ld >= n");
    const double *d = d_d;
    if (d_dsc_out) {
        k_diag_scale<<<(n + 255) / 256, 256, 0, S(stream)>>>(d_Z, n, ld, d_dsc_out);
        M25_LAUNCH_CHECK("k_diag_scale");
        d = d_dsc_out;
    }
    M25_REQUIRE(d, "m25_equilibrate: scales or an output for them");
    dim3 grid((unsigned)std::min<long>((n + 255) / 256, 64), (unsigned)n);
    k_equilibrate<<<grid, 256, 0, S(stream)>>>(d_Z, n, ld, d, d_Z64);
    M25_LAUNCH_CHECK("k_equilibrate");
    return M25_OK;
}

// the same for a complex64 Z (the mixed-precision path fills Z in complex64 directly): scales from its diagonal
extern "C" int m25_equilibrate_c64(float *d_Z, long n, long ld, double *d_dsc_out, void *stream)
{
    M25_REQUIRE(d_Z && d_dsc_out && ld >= n, "m25_equilibrate_c64: Z, scales, ld >= n");
    k_diag_scale_c64<<<(n + 255) / 256, 256, 0, S(stream)>>>(d_Z, n, ld, d_dsc_out);
    M25_LAUNCH_CHECK("k_diag_scale_c64");
    dim3 grid((unsigned)std::min<long>((n + 255) / 256, 64), (unsigned)n);
    k_equilibrate_c64<<<grid, 256, 0, S(stream)>>>(d_Z, n, ld, d_dsc_out);
    M25_LAUNCH_CHECK("k_equilibrate_c64");
    return M25_OK;
}
