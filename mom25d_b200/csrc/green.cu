// green.cu - the layered-media Green tables on the GPU: the stack's transmission-line network at the points of the
// Sommerfeld contour, the Hankel transform to the radial grid (one block per radius, Bessel values never stored),
// the not-a-knot cubic spline to the fine uniform grid the fill interpolates, and the via kernels' spectra.
// Restates multilayer.py:183-318 and via.py:36-235 (cited per kernel); complex128 throughout.
#include "common.cuh"

#define M25_MAX_LAYERS 8
#define M25_C0 299792458.0
#define M25_MU0 (4e-7 * 3.14159265358979323846)
#define M25_EPS0 (1.0 / (M25_MU0 * M25_C0 * M25_C0))

// ---- complex elementary functions (principal branches) ----------------------------------------------------------------
__device__ __forceinline__ zd zsqrt(zd z)
{
    // csqrt: the root with non-negative real part, computed without cancellation
    double a = z.x, b = z.y;
    if (a == 0 && b == 0) return mk<double>(0, b);
    double t = sqrt(0.5 * (fabs(a) + hypot(a, b)));
    if (a >= 0) return mk<double>(t, b / (2 * t));
    return mk<double>(fabs(b) / (2 * t), copysign(t, b));
}
__device__ __forceinline__ zd zexp(zd z)
{
    double e = exp(z.x), s, c;
    sincos(z.y, &s, &c);
    return mk<double>(e * c, e * s);
}
__device__ __forceinline__ zd zlog(zd z) { return mk<double>(log(hypot(z.x, z.y)), atan2(z.y, z.x)); }
__device__ __forceinline__ zd zcos(zd z)
{
    double s, c;
    sincos(z.x, &s, &c);
    return mk<double>(c * cosh(z.y), -s * sinh(z.y));
}
__device__ __forceinline__ zd zsin(zd z)
{
    double s, c;
    sincos(z.x, &s, &c);
    return mk<double>(s * cosh(z.y), c * sinh(z.y));
}
__device__ __forceinline__ zd zdiv(zd a, zd b) { return cdiv<double>(a, b); }
__device__ __forceinline__ zd zi(zd a) { return mk<double>(-a.y, a.x); }          // 1j * a
__device__ __forceinline__ zd zmi(zd a) { return mk<double>(a.y, -a.x); }         // -1j * a
__device__ __forceinline__ double zabs(zd a) { return hypot(a.x, a.y); }

// ---- the stack (multilayer.py:90-250) -------------------------------------------------------------------------------
struct Stack {
    int N;                              // layers
    int top_open;                       // 1: half-space above (top_eps); 0: PEC cover on interface N
    double h[M25_MAX_LAYERS];
    zd eps[M25_MAX_LAYERS + 2];         // eps[j], j = 1..N the layers, N + 1 the half-space above
};

// The network of one mode at one kr (multilayer.py:183-219): Y0, tn, sc per layer 1..N, Yd, Yu per interface.
struct Net {
    zd Y0[M25_MAX_LAYERS + 1], tn[M25_MAX_LAYERS + 1], sc[M25_MAX_LAYERS + 1];
    zd Yd[M25_MAX_LAYERS + 1], Yu[M25_MAX_LAYERS + 1];
};

__device__ void y0_of(const Stack &st, zd kr, double w, zd e, bool te, zd &Y0, zd &kz)
{
    const double k0 = w / M25_C0;
    zd kr2 = kr * kr;
    zd arg = kr2 - e * (k0 * k0);
    kz = zmi(zsqrt(arg));                                 // -1j sqrt(kr^2 - k0^2 e)
    if (te) Y0 = kz / (w * M25_MU0);
    else Y0 = zdiv(e * (w * M25_EPS0), kz);
}

__device__ void network(const Stack &st, zd kr, double w, bool te, Net &n)
{
    const int N = st.N;
    for (int j = 1; j <= N; ++j) {
        zd kz;
        y0_of(st, kr, w, st.eps[j], te, n.Y0[j], kz);
        zd th = kz * st.h[j - 1];
        zd E = zexp(mk<double>(2 * th.y, -2 * th.x));    // exp(-2j th)
        zd one = mk<double>(1, 0);
        n.tn[j] = zdiv(zmi(one - E), one + E);             // -1j (1 - E) / (1 + E)
        n.sc[j] = zdiv(zexp(mk<double>(th.y, -th.x)) * 2.0, one + E);   // 2 exp(-1j th) / (1 + E)
    }
    n.Yd[1] = zdiv(zmi(n.Y0[1]), n.tn[1]);                // shorted by the ground plane
    for (int k = 2; k <= N; ++k)
        n.Yd[k] = n.Y0[k] * zdiv(n.Yd[k - 1] + zi(n.Y0[k] * n.tn[k]), n.Y0[k] + zi(n.Yd[k - 1] * n.tn[k]));
    int kstart;
    if (st.top_open) {
        zd kz;
        y0_of(st, kr, w, st.eps[N + 1], te, n.Yu[N], kz);
        kstart = N;
    } else {
        n.Yu[N - 1] = zdiv(zmi(n.Y0[N]), n.tn[N]);
        kstart = N - 1;
    }
    for (int k = kstart; k > 1; --k)
        n.Yu[k - 1] = n.Y0[k] * zdiv(n.Yu[k] + zi(n.Y0[k] * n.tn[k]), n.Y0[k] + zi(n.Yu[k] * n.tn[k]));
}

__device__ __forceinline__ bool is_pec(const Stack &st, int k) { return k == 0 || (k == st.N && !st.top_open); }

// multilayer.py:234-245: voltage at o for a unit shunt current at s
__device__ zd voltage(const Stack &st, const Net &n, int o, int s)
{
    if (is_pec(st, o) || is_pec(st, s)) return mk<double>(0, 0);
    zd v = zdiv(mk<double>(1, 0), n.Yu[s] + n.Yd[s]);
    for (int k = s + 1; k <= o; ++k)
        v = zdiv(v * n.sc[k], mk<double>(1, 0) + zi(zdiv(n.Yu[k], n.Y0[k]) * n.tn[k]));
    for (int k = s; k > o; --k)
        v = zdiv(v * n.sc[k], mk<double>(1, 0) + zi(zdiv(n.Yd[k - 1], n.Y0[k]) * n.tn[k]));
    return v;
}

// multilayer.py:247-250 (spectral), then the singular parts taken out (multilayer.py:287-289):
// G - sum c 2 pi exp(-kr d) / kr over the extracted (d, cA, cq)
struct PairSpec {
    int o, s, next;          // interfaces; number of extracted parts
    double d[2];
    zd cA[2], cq[2];
};

__global__ void k_spectral_tables(const double *kr_, int npts, double w, Stack st, const PairSpec *pairs, int npair,
                                  double *GA, double *GQ)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= npts) return;
    zd kr = ldc<double>(kr_, k);
    Net nh, ne;
    network(st, kr, w, true, nh);
    network(st, kr, w, false, ne);
    zd jw = mk<double>(0, w);
    for (int p = 0; p < npair; ++p) {
        PairSpec ps = pairs[p];
        zd Vh = voltage(st, nh, ps.o, ps.s), Ve = voltage(st, ne, ps.o, ps.s);
        zd ga = zdiv(Vh, jw), gq = zdiv(jw * (Ve - Vh), kr * kr);
        for (int j = 0; j < ps.next; ++j) {
            zd e = zdiv(zexp(mk<double>(-kr.x * ps.d[j], -kr.y * ps.d[j])) * (2 * 3.14159265358979323846), kr);
            ga = ga - ps.cA[j] * e;
            gq = gq - ps.cq[j] * e;
        }
        stc<double>(GA, (size_t)p * npts + k, ga);
        stc<double>(GQ, (size_t)p * npts + k, gq);
    }
}

// Spectral G_A, G_q of a pair at single points (the singular coefficients' large-kr limits, multilayer.py:271-287)
__global__ void k_spectral_points(const double *kr_, const double *w_, int npts, Stack st, int o, int s, double *ga_,
                                  double *gq_)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= npts) return;
    zd kr = ldc<double>(kr_, k);
    double w = w_[k];
    Net nh, ne;
    network(st, kr, w, true, nh);
    network(st, kr, w, false, ne);
    zd jw = mk<double>(0, w);
    zd Vh = voltage(st, nh, o, s), Ve = voltage(st, ne, o, s);
    stc<double>(ga_, k, zdiv(Vh, jw));
    stc<double>(gq_, k, zdiv(jw * (Ve - Vh), kr * kr));
}

// ---- via spectra (via.py:127-235): D(k, span) and R(span_m, span_n) ------------------------------------------------
// TM voltages V[s][i] for every source interface s = 1..N (open top) / 1..N-1 (PEC cover) (via.py:127-146)
__device__ void tm_voltages(const Stack &st, const Net &ne, zd V[M25_MAX_LAYERS + 1][M25_MAX_LAYERS + 1])
{
    const int N = st.N;
    for (int s = 0; s <= N; ++s)
        for (int i = 0; i <= N; ++i) V[s][i] = mk<double>(0, 0);
    for (int s = 1; s <= N; ++s) {
        if (is_pec(st, s)) continue;
        V[s][s] = zdiv(mk<double>(1, 0), ne.Yu[s] + ne.Yd[s]);
        for (int k = s + 1; k <= N; ++k)
            V[s][k] = is_pec(st, k) ? mk<double>(0, 0) :
                      zdiv(V[s][k - 1] * ne.sc[k], mk<double>(1, 0) + zi(zdiv(ne.Yu[k], ne.Y0[k]) * ne.tn[k]));
        for (int k = s; k > 0; --k)
            V[s][k - 1] = is_pec(st, k - 1) ? mk<double>(0, 0) :
                          zdiv(V[s][k] * ne.sc[k], mk<double>(1, 0) + zi(zdiv(ne.Yd[k - 1], ne.Y0[k]) * ne.tn[k]));
    }
}

struct ViaSpecReq {
    int nd, nr;                 // D specs (k, span) then R specs (span_m, span_n)
    int dk[32], dspan[32][2];
    int rm[32][2], rn[32][2];
};

__global__ void k_via_spectra(const double *kr_, int npts, double w, Stack st, ViaSpecReq rq, double *out)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= npts) return;
    const int N = st.N;
    zd kr = ldc<double>(kr_, k);
    Net nh, ne;
    network(st, kr, w, true, nh);
    network(st, kr, w, false, ne);
    zd V[M25_MAX_LAYERS + 1][M25_MAX_LAYERS + 1];
    tm_voltages(st, ne, V);
    const double k0 = w / M25_C0;
    zd kz2[M25_MAX_LAYERS + 1];
    for (int j = 1; j <= N; ++j) kz2[j] = st.eps[j] * (k0 * k0) - kr * kr;
    zd jw = mk<double>(0, w);
    auto dV = [&](int i, int s) -> zd { return is_pec(st, s) ? mk<double>(0, 0) : V[s][i] - V[s][i - 1]; };
    auto gq = [&](int a, int b) -> zd {
        if (is_pec(st, a) || is_pec(st, b)) return mk<double>(0, 0);
        int lo = a < b ? a : b, hi = a < b ? b : a;
        zd Vh = voltage(st, nh, lo, hi), Ve = voltage(st, ne, lo, hi);
        return zdiv(jw * (Ve - Vh), kr * kr);
    };
    int row = 0;
    for (int r = 0; r < rq.nd; ++r, ++row) {                 // via.py:205-210
        int kk = rq.dk[r], kb = rq.dspan[r][0], kt = rq.dspan[r][1];
        zd spec = mk<double>(0, 0);
        for (int j = kb + 1; j <= kt; ++j) spec += zdiv(dV(j, kk), kz2[j]);
        spec = spec - zdiv(gq(kk, kb) * 1.0, jw);
        spec = spec + zdiv(gq(kk, kt), jw);
        stc<double>(out, (size_t)row * npts + k, spec);
    }
    zd kr2 = kr * kr;
    for (int r = 0; r < rq.nr; ++r, ++row) {                 // via.py:215-220 (P without the homogeneous term)
        int mb = rq.rm[r][0], mt = rq.rm[r][1], nb = rq.rn[r][0], nt = rq.rn[r][1];
        zd spec = mk<double>(0, 0);
        for (int i = mb + 1; i <= mt; ++i)
            for (int j = nb + 1; j <= nt; ++j)
                spec += zdiv(kr2, kz2[i] * kz2[j]) * (dV(i, j) - dV(i, j - 1));
        int ka[2] = {mb, mt}, kb2[2] = {nb, nt};
        double da[2] = {1.0, -1.0};
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b)
                spec = spec - zdiv(gq(ka[a], kb2[b]) * (da[a] * da[b]), jw);
        stc<double>(out, (size_t)row * npts + k, spec);
    }
}

// ---- complex Bessel J_n (mom25d_core.cpp:1510-1543: power series to |z| = 14, Hankel's expansion beyond) -------------
__device__ zd jn_complex(int n, zd z)
{
    const double PI = 3.14159265358979323846;
    const double az = zabs(z);
    if (az <= 14.0) {
        const zd h = z * 0.5, mh2 = mk<double>(0, 0) - h * h;
        zd term = n == 0 ? mk<double>(1, 0) : n == 1 ? h : (h * h) * 0.5;
        zd sum = term;
        double big = zabs(term);
        for (int k = 1; k < 300; ++k) {
            term = term * (mh2 / ((double)k * (double)(k + n)));
            sum += term;
            const double at = zabs(term);
            big = fmax(big, at);
            if (k > az && at <= 1e-18 * big) break;
        }
        return sum;
    }
    const double mu = 4.0 * n * n;
    const zd iz = zdiv(mk<double>(1, 0), z), chi = z - mk<double>((0.5 * n + 0.25) * PI, 0);
    zd P = mk<double>(1, 0), Q = mk<double>(0, 0), t = mk<double>(1, 0);
    double prev = 1.0;
    for (int k = 1; k < 80; ++k) {
        const double m = 2.0 * k - 1.0;
        const zd nt = (t * ((mu - m * m) / (8.0 * k))) * iz;
        const double at = zabs(nt);
        if (at >= prev) break;
        t = nt; prev = at;
        const double sg = ((k / 2) & 1) ? -1.0 : 1.0;
        if (k & 1) Q += t * sg; else P += t * sg;
        if (at < 1e-17) break;
    }
    return zsqrt(zdiv(mk<double>(2.0, 0), z * PI)) * (P * zcos(chi) - Q * zsin(chi));
}

__global__ void k_bessel_jn(int n, const double *z, long count, double *out)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < count) stc<double>(out, i, jn_complex(n, ldc<double>(z, i)));
}

// ---- K0 of complex argument (the via kernels' homogeneous term, via.py:228-235): power series for |z| <= 14,
// the asymptotic expansion (to its smallest term) beyond -------------------------------------------------------------
__device__ zd k0_complex(zd z)
{
    const double PI = 3.14159265358979323846, GAMMA = 0.57721566490153286061;
    const double az = zabs(z);
    if (az <= 14.0) {
        zd q = (z * z) * 0.25;                               // z^2 / 4
        zd lg = zlog(z * 0.5) + mk<double>(GAMMA, 0);
        zd term = mk<double>(1, 0), I0 = term, S = mk<double>(0, 0);
        double H = 0, big = 1;
        for (int k = 1; k < 300; ++k) {
            term = term * (q / ((double)k * (double)k));
            H += 1.0 / k;
            I0 += term;
            S += term * H;
            double at = zabs(term) * fmax(1.0, H);
            big = fmax(big, at);
            if (k > az && at <= 1e-18 * big) break;
        }
        return S - lg * I0;
    }
    // sqrt(pi / 2z) e^-z sum_k a_k / z^k, a_k = prod (-(2j-1)^2) / (k! 8^k)
    zd iz = zdiv(mk<double>(1, 0), z);
    zd sum = mk<double>(1, 0), t = mk<double>(1, 0);
    double prev = 1.0;
    for (int k = 1; k < 80; ++k) {
        double m = 2.0 * k - 1.0;
        zd nt = (t * (-(m * m) / (8.0 * k))) * iz;
        double at = zabs(nt);
        if (at >= prev) break;
        t = nt; prev = at;
        sum += t;
        if (at < 1e-17) break;
    }
    return zsqrt(zdiv(mk<double>(PI * 0.5, 0), z)) * zexp(mk<double>(-z.x, -z.y)) * sum;
}

// homog (via.py:228-235): sum over the shared layers j of jw mu0 h_j / 2pi K0(1j kj rho), kj = -sqrt(k_j^2) when
// its imaginary part is positive. layer_mask bit j: layer j is shared.
__global__ void k_via_homog(const double *rho, int n, double w, Stack st, unsigned layer_mask, double *out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double k0 = w / M25_C0;
    zd acc = mk<double>(0, 0);
    for (int j = 1; j <= st.N; ++j) {
        if (!(layer_mask & (1u << j))) continue;
        zd kj = zsqrt(st.eps[j] * (k0 * k0));
        if (kj.y > 0) kj = mk<double>(-kj.x, -kj.y);
        zd K = k0_complex(zi(kj) * rho[i]);
        acc += K * mk<double>(0, w * M25_MU0 * st.h[j - 1] / (2 * 3.14159265358979323846));
    }
    stc<double>(out, i, acc);
}

// ---- Hankel transform (via.py:90-108): out[s, i] = (1/2pi) sum_k J0(rho_i kr_k) W[s, k] kr_k dk_k -------------------
// One block per radius; the contour split over the threads (J0 of a real argument: the CUDA math library's j0;
// on the lifted part the complex series above); then a block reduction per spectrum.
// RAW: the bare sum over real kr (hankel_real, mom25d_core.cpp:1430-1454): out[s, i] = sum_k J0(rho_i kr_k) W[s, k],
// kr_ real f64[npts], no dk, no 1 / 2 pi.
template <int NS, bool RAW = false>
__global__ void __launch_bounds__(256) k_hankel(const double *kr_, const double *dk_, int npts, const double *W, int ns,
                                                const double *rho, double *out, int nr)
{
    const int i = blockIdx.x;
    if (i >= nr) return;
    const double r = rho[i];
    zd acc[NS];
    for (int s = 0; s < NS; ++s) acc[s] = mk<double>(0, 0);
    for (int k = threadIdx.x; k < npts; k += blockDim.x) {
        zd f;
        if (RAW) {
            f = mk<double>(j0(r * kr_[k]), 0);
        } else {
            zd kr = ldc<double>(kr_, k), dk = ldc<double>(dk_, k);
            zd J = fabs(kr.y) < 1e-300 ? mk<double>(j0(r * kr.x), 0) : jn_complex(0, kr * r);
            f = J * (kr * dk);
        }
        for (int s = 0; s < NS; ++s)
            if (s < ns) acc[s] += f * ldc<double>(W, (size_t)s * npts + k);
    }
    __shared__ zd red[256 / 32][NS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int s = 0; s < NS; ++s) {
        double x = acc[s].x, y = acc[s].y;
        for (int o = 16; o; o >>= 1) { x += __shfl_xor_sync(0xffffffffu, x, o); y += __shfl_xor_sync(0xffffffffu, y, o); }
        if (lane == 0) red[wid][s] = mk<double>(x, y);
    }
    __syncthreads();
    if (threadIdx.x < NS && threadIdx.x < ns) {
        zd t = mk<double>(0, 0);
        for (int j = 0; j < (int)(blockDim.x / 32); ++j) t += red[j][threadIdx.x];
        stc<double>(out, (size_t)threadIdx.x * nr + i, RAW ? t : t * (1.0 / (2 * 3.14159265358979323846)));
    }
}

// ---- not-a-knot cubic spline to a uniform grid (via.py:111-123; SciPy CubicSpline and PPoly evaluation) ------------
// One block per spectrum: thread 0 solves the tridiagonal system for the slopes (Thomas), the block evaluates.
// Out of range points extrapolate with the end pieces, as PPoly does.
template <typename OutR>
__global__ void __launch_bounds__(256) k_spline_uniform(const double *x, const double *y, int n, double dx, int nfine,
                                                        OutR *out, long out_stride, long out_offset, int interleave)
{
    extern __shared__ unsigned char smem_raw[];
    zd *c = reinterpret_cast<zd *>(smem_raw);              // 4 (n - 1) coefficients
    zd *s = c + 4 * (n - 1);                               // slopes, n
    double *xs = reinterpret_cast<double *>(s + n);        // x, n
    const int row = blockIdx.x;
    const double *yr = y + 2 * (size_t)row * n;
    for (int i = threadIdx.x; i < n; i += blockDim.x) xs[i] = x[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        // the banded system of scipy.interpolate.CubicSpline, not-a-knot at both ends
        // (a: sub-diagonal, b: diagonal, cc: super-diagonal, rhs)
        zd *rhs = c;                                        // scratch inside c before the coefficients are written
        double *a = reinterpret_cast<double *>(c + n), *b = a + n, *cc = b + n;
        auto dxi = [&](int i) { return xs[i + 1] - xs[i]; };
        auto slope = [&](int i) { return (ldc<double>(yr, i + 1) - ldc<double>(yr, i)) / dxi(i); };
        for (int i = 1; i < n - 1; ++i) {
            b[i] = 2 * (dxi(i - 1) + dxi(i));
            cc[i] = dxi(i - 1);
            a[i] = dxi(i);
            rhs[i] = (slope(i - 1) * dxi(i) + slope(i) * dxi(i - 1)) * 3.0;
        }
        {
            double d = xs[2] - xs[0];
            b[0] = dxi(1); cc[0] = d; a[0] = 0;
            rhs[0] = (slope(0) * ((dxi(0) + 2 * d) * dxi(1)) + slope(1) * (dxi(0) * dxi(0))) / d;
            d = xs[n - 1] - xs[n - 3];
            b[n - 1] = dxi(n - 3); a[n - 1] = d; cc[n - 1] = 0;
            rhs[n - 1] = (slope(n - 3) * (dxi(n - 2) * dxi(n - 2)) + slope(n - 2) * ((2 * d + dxi(n - 2)) * dxi(n - 3))) / d;
        }
        // Thomas forward sweep: row i = a[i] s[i-1] + b[i] s[i] + cc[i] s[i+1]
        for (int i = 1; i < n; ++i) {
            double m = a[i] / b[i - 1];
            b[i] -= m * cc[i - 1];
            rhs[i] = rhs[i] - rhs[i - 1] * m;
        }
        s[n - 1] = rhs[n - 1] / b[n - 1];
        for (int i = n - 2; i >= 0; --i) s[i] = (rhs[i] - s[i + 1] * cc[i]) / b[i];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n - 1; i += blockDim.x) {
        double h = xs[i + 1] - xs[i];
        zd sl = (ldc<double>(yr, i + 1) - ldc<double>(yr, i)) / h;
        zd t = (s[i] + s[i + 1] - sl * 2.0) / h;
        c[4 * i + 0] = t / h;
        c[4 * i + 1] = (sl - s[i]) / h - t;
        c[4 * i + 2] = s[i];
        c[4 * i + 3] = ldc<double>(yr, i);
    }
    __syncthreads();
    const double x0 = xs[0], xn = xs[n - 1];
    for (int j = threadIdx.x; j < nfine; j += blockDim.x) {
        double xf = (j == nfine - 1) ? xn : (double)j * dx;      // numpy.linspace: j * step, the last point exact
        // the interval: x[i] <= xf < x[i+1] (the last one closed), by bisection
        int lo = 0, hi = n - 2;
        if (xf <= x0) lo = 0;
        else if (xf >= xs[n - 2]) lo = n - 2;
        else {
            while (hi - lo > 1) {
                int mid = (lo + hi) >> 1;
                if (xs[mid] <= xf) lo = mid; else hi = mid;
            }
            if (xs[hi] <= xf) lo = hi;
        }
        double hh = xf - xs[lo];
        // PPoly's evaluate_poly1: c3 + c2 h + c1 h^2 + c0 h^3, powers accumulated
        zd res = c[4 * lo + 3];
        double z = hh;
        res += c[4 * lo + 2] * z; z *= hh;
        res += c[4 * lo + 1] * z; z *= hh;
        res += c[4 * lo + 0] * z;
        size_t o = (size_t)row * out_stride + out_offset + (size_t)j * interleave;
        out[2 * o] = (OutR)res.x;
        out[2 * o + 1] = (OutR)res.y;
    }
}

// ======================================================================================================================
static inline cudaStream_t S(void *s) { return (cudaStream_t)s; }

static int make_stack(int nl, const double *h_h, const double *h_eps, int top_open, const double *h_top_eps, Stack &st)
{
    M25_REQUIRE(nl >= 1 && nl < M25_MAX_LAYERS, "a stack of 1 to 7 layers");
    st.N = nl;
    st.top_open = top_open;
    for (int j = 0; j < nl; ++j) {
        st.h[j] = h_h[j];
        st.eps[j + 1] = mk<double>(h_eps[2 * j], h_eps[2 * j + 1]);
    }
    st.eps[nl + 1] = top_open ? mk<double>(h_top_eps[0], h_top_eps[1]) : mk<double>(1, 0);
    st.eps[0] = mk<double>(1, 0);
    return M25_OK;
}

extern "C" int m25_spectral(const double *d_kr, int npts, double w, int nl, const double *h_h, const double *h_eps,
                            int top_open, const double *h_top_eps, int npair, const int *h_o, const int *h_s,
                            double *d_GA, double *d_GQ, void *stream)
{
    // the plain spectral kernels of npair pairs (no extraction): used by the table builder through m25_green_spectra
    Stack st;
    int rc = make_stack(nl, h_h, h_eps, top_open, h_top_eps, st);
    if (rc) return rc;
    M25_REQUIRE(npair >= 0 && npair <= 64, "m25_spectral: at most 64 pairs");
    PairSpec ps[64];
    for (int i = 0; i < npair; ++i) { ps[i].o = h_o[i]; ps[i].s = h_s[i]; ps[i].next = 0; }
    PairSpec *d_ps;
    M25_CHECK(cudaMallocAsync(&d_ps, sizeof(PairSpec) * (npair ? npair : 1), S(stream)));
    M25_CHECK(cudaMemcpyAsync(d_ps, ps, sizeof(PairSpec) * npair, cudaMemcpyHostToDevice, S(stream)));
    k_spectral_tables<<<(npts + 127) / 128, 128, 0, S(stream)>>>(d_kr, npts, w, st, d_ps, npair, d_GA, d_GQ);
    cudaError_t le = cudaGetLastError();
    cudaError_t fe = cudaFreeAsync(d_ps, S(stream));
    if (le != cudaSuccess) return m25_cuda_status(le, "k_spectral_tables");
    if (fe != cudaSuccess) return m25_cuda_status(fe, "cudaFreeAsync");
    return M25_OK;
}

// Tables with their singular parts taken out: per pair (o, s) the extracted (d, cA, cq) list (host arrays of
// npair x 2 entries; next[i] of them used). The extraction coefficients themselves come from
// m25_spectral_points (their large-kr limits are computed on the GPU by the host code, multilayer.py:271-287).
extern "C" int m25_spectral_extracted(const double *d_kr, int npts, double w, int nl, const double *h_h,
                                      const double *h_eps, int top_open, const double *h_top_eps, int npair,
                                      const int *h_o, const int *h_s, const int *h_next, const double *h_d,
                                      const double *h_cA, const double *h_cq, double *d_GA, double *d_GQ,
                                      void *d_pairs_scratch, void *stream)
{
    Stack st;
    int rc = make_stack(nl, h_h, h_eps, top_open, h_top_eps, st);
    if (rc) return rc;
    M25_REQUIRE(npair >= 1 && npair <= 64, "m25_spectral_extracted: 1 to 64 pairs");
    M25_REQUIRE(d_pairs_scratch, "m25_spectral_extracted: scratch of 64 pair records");
    PairSpec ps[64];
    for (int i = 0; i < npair; ++i) {
        ps[i].o = h_o[i]; ps[i].s = h_s[i]; ps[i].next = h_next[i];
        for (int j = 0; j < 2; ++j) {
            ps[i].d[j] = h_d[2 * i + j];
            ps[i].cA[j] = mk<double>(h_cA[4 * i + 2 * j], h_cA[4 * i + 2 * j + 1]);
            ps[i].cq[j] = mk<double>(h_cq[4 * i + 2 * j], h_cq[4 * i + 2 * j + 1]);
        }
    }
    M25_CHECK(cudaMemcpyAsync(d_pairs_scratch, ps, sizeof(PairSpec) * npair, cudaMemcpyHostToDevice, S(stream)));
    M25_CHECK(cudaStreamSynchronize(S(stream)));      // ps is a stack buffer: the copy must land first
    k_spectral_tables<<<(npts + 127) / 128, 128, 0, S(stream)>>>(d_kr, npts, w, st, (const PairSpec *)d_pairs_scratch,
                                                                 npair, d_GA, d_GQ);
    M25_LAUNCH_CHECK("k_spectral_tables");
    return M25_OK;
}

extern "C" size_t m25_pair_record_bytes(void) { return sizeof(PairSpec) * 64; }

extern "C" int m25_spectral_points(const double *d_kr, const double *d_w, int npts, int nl, const double *h_h,
                                   const double *h_eps, int top_open, const double *h_top_eps, int o, int s,
                                   double *d_ga, double *d_gq, void *stream)
{
    Stack st;
    int rc = make_stack(nl, h_h, h_eps, top_open, h_top_eps, st);
    if (rc) return rc;
    k_spectral_points<<<(npts + 127) / 128, 128, 0, S(stream)>>>(d_kr, d_w, npts, st, o, s, d_ga, d_gq);
    M25_LAUNCH_CHECK("k_spectral_points");
    return M25_OK;
}

extern "C" int m25_via_spectra(const double *d_kr, int npts, double w, int nl, const double *h_h, const double *h_eps,
                               int top_open, const double *h_top_eps, int nd, const int *h_dk, const int *h_dspan,
                               int nr, const int *h_rm, const int *h_rn, double *d_out, void *stream)
{
    Stack st;
    int rc = make_stack(nl, h_h, h_eps, top_open, h_top_eps, st);
    if (rc) return rc;
    M25_REQUIRE(nd <= 32 && nr <= 32, "m25_via_spectra: at most 32 D and 32 R spectra");
    ViaSpecReq rq;
    rq.nd = nd; rq.nr = nr;
    for (int i = 0; i < nd; ++i) { rq.dk[i] = h_dk[i]; rq.dspan[i][0] = h_dspan[2 * i]; rq.dspan[i][1] = h_dspan[2 * i + 1]; }
    for (int i = 0; i < nr; ++i) {
        rq.rm[i][0] = h_rm[2 * i]; rq.rm[i][1] = h_rm[2 * i + 1];
        rq.rn[i][0] = h_rn[2 * i]; rq.rn[i][1] = h_rn[2 * i + 1];
    }
    k_via_spectra<<<(npts + 127) / 128, 128, 0, S(stream)>>>(d_kr, npts, w, st, rq, d_out);
    M25_LAUNCH_CHECK("k_via_spectra");
    return M25_OK;
}

extern "C" int m25_via_homog(const double *d_rho, int n, double w, int nl, const double *h_h, const double *h_eps,
                             int top_open, const double *h_top_eps, unsigned layer_mask, double *d_out, void *stream)
{
    Stack st;
    int rc = make_stack(nl, h_h, h_eps, top_open, h_top_eps, st);
    if (rc) return rc;
    if (!n) return M25_OK;
    k_via_homog<<<(n + 127) / 128, 128, 0, S(stream)>>>(d_rho, n, w, st, layer_mask, d_out);
    M25_LAUNCH_CHECK("k_via_homog");
    return M25_OK;
}

extern "C" int m25_hankel(const double *d_kr, const double *d_dk, int npts, const double *d_W, int ns,
                          const double *d_rho, int nr, double *d_out, void *stream)
{
    M25_REQUIRE(ns >= 1 && ns <= 16, "m25_hankel: 1 to 16 spectra a call");
    if (!nr) return M25_OK;
    if (ns <= 4) k_hankel<4><<<nr, 256, 0, S(stream)>>>(d_kr, d_dk, npts, d_W, ns, d_rho, d_out, nr);
    else if (ns <= 8) k_hankel<8><<<nr, 256, 0, S(stream)>>>(d_kr, d_dk, npts, d_W, ns, d_rho, d_out, nr);
    else k_hankel<16><<<nr, 256, 0, S(stream)>>>(d_kr, d_dk, npts, d_W, ns, d_rho, d_out, nr);
    M25_LAUNCH_CHECK("k_hankel");
    return M25_OK;
}

extern "C" int m25_hankel_real(const double *d_rho, int nr, const double *d_kr, int nk, const double *d_W, int ns,
                               double *d_out, void *stream)
{
    M25_REQUIRE(ns >= 1 && ns <= 16, "m25_hankel_real: 1 to 16 rows of W a call");
    if (!nr) return M25_OK;
    if (ns <= 4) k_hankel<4, true><<<nr, 256, 0, S(stream)>>>(d_kr, nullptr, nk, d_W, ns, d_rho, d_out, nr);
    else if (ns <= 8) k_hankel<8, true><<<nr, 256, 0, S(stream)>>>(d_kr, nullptr, nk, d_W, ns, d_rho, d_out, nr);
    else k_hankel<16, true><<<nr, 256, 0, S(stream)>>>(d_kr, nullptr, nk, d_W, ns, d_rho, d_out, nr);
    M25_LAUNCH_CHECK("k_hankel");
    return M25_OK;
}

extern "C" int m25_spline_uniform(const double *d_x, const double *d_y, int ns, int n, double dx, int nfine, void *d_out,
                                  int single, long out_stride, long out_offset_elems, int out_interleave, void *stream)
{
    M25_REQUIRE(n >= 4 && ns >= 1 && nfine >= 2, "m25_spline_uniform: n >= 4 points");
    size_t smem = sizeof(zd) * (4 * (size_t)(n - 1) + n) + sizeof(double) * n;
    M25_REQUIRE(smem <= 200 * 1024, "m25_spline_uniform: too many knots");
    if (smem > 48 * 1024) {
        M25_CHECK(cudaFuncSetAttribute(k_spline_uniform<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        M25_CHECK(cudaFuncSetAttribute(k_spline_uniform<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    if (single)
        k_spline_uniform<float><<<ns, 256, smem, S(stream)>>>(d_x, d_y, n, dx, nfine, (float *)d_out, out_stride,
                                                               out_offset_elems, out_interleave);
    else
        k_spline_uniform<double><<<ns, 256, smem, S(stream)>>>(d_x, d_y, n, dx, nfine, (double *)d_out, out_stride,
                                                                out_offset_elems, out_interleave);
    M25_LAUNCH_CHECK("k_spline_uniform");
    return M25_OK;
}

extern "C" int m25_bessel_jn_complex(int order, const double *d_z, long count, double *d_out, void *stream)
{
    M25_REQUIRE(order >= 0 && order <= 2, "m25_bessel_jn_complex: order 0, 1 or 2");
    if (!count) return M25_OK;
    k_bessel_jn<<<(count + 255) / 256, 256, 0, S(stream)>>>(order, d_z, count, d_out);
    M25_LAUNCH_CHECK("k_bessel_jn");
    return M25_OK;
}
