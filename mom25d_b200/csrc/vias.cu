// vias.cu - the via rows and columns of Z on the GPU (mom25d sim.py:816-872 _via_blocks, fast.py:489-504
// _fan_columns): fan-distributed end charges through G_q, the smooth via -> strip kernel D tested with the RWG
// divergence, the via-via block C, written straight into the bordered N x N matrix.
#include "common.cuh"

static inline cudaStream_t S(void *s) { return (cudaStream_t)s; }

// QF[P[k], col[k]] += qcorr[pair[k]]: the near pairs' G_q moment corrections on the fan columns (fast.py:501-503)
__global__ void k_qcorr_scatter(double *QF, int nf, const int *pair, const int *row, const int *col, int n,
                                const double *qcorr)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    zd v = ldc<double>(qcorr, pair[k]);
    size_t o = (size_t)row[k] * nf + col[k];
    atomicAdd(QF + 2 * o, v.x);
    atomicAdd(QF + 2 * o + 1, v.y);
}

// T[t, n] = sum over chain n's fan entries (j, weight) of QF[t, j] weight  (dF as CSR by chain)
__global__ void k_fan_T(const double *QF, int Nt, int nf, const int *ptr, const int *fj, const double *fw, int Nv,
                        double *T)
{
    long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (idx >= (long)Nt * Nv) return;
    int t = idx / Nv, n = idx % Nv;
    zd acc = mk<double>(0, 0);
    for (int k = ptr[n]; k < ptr[n + 1]; ++k) acc += ldc<double>(QF, (size_t)t * nf + fj[k]) * fw[k];
    stc<double>(T, idx, acc);
}

// c[t, n] = sum_q D_{tab[lt[t], span[n]]}(|P6[t, q] - V_n|) W6[t, q] (radial_table_sum per layer and span,
// mom25d_core.cpp:1269-1298; the tables' lerp of via.Table1D)
__global__ void k_radial_layers(const double *P6, const double *W6, const int *lt, int Nt, const double *vx,
                                const double *vy, const int *span_of, int Nv, const double *D, const int *dtab,
                                int nspan, long nfine, double dr, double *c)
{
    long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (idx >= (long)Nt * Nv) return;
    int t = idx / Nv, n = idx % Nv;
    const double *tb = D + 2 * (size_t)dtab[lt[t] * nspan + span_of[n]] * nfine;
    const double top = (double)nfine - 1.000001;
    zd acc = mk<double>(0, 0);
    for (int q = 0; q < 6; ++q) {
        const double rx = P6[12 * (size_t)t + 2 * q] - vx[n], ry = P6[12 * (size_t)t + 2 * q + 1] - vy[n];
        double u = fmin(hypot(rx, ry) / dr, top);
        long i = (long)u;
        double f = u - (double)i;
        acc += (ldc<double>(tb, i) * (1.0 - f) + ldc<double>(tb, i + 1) * f) * W6[6 * (size_t)t + q];
    }
    stc<double>(c, idx, acc);
}

// B[e, n] = 2 alpha+ (T[tp, n] / jw + c[tp, n]) + 2 alpha- (T[tm, n] / jw + c[tm, n]) into Z[e, Ne + n] and its
// transpose into Z[Ne + n, e] (sim.py:856-858: B = D^T (T / jw + c))
// where the border goes: the complex128 Z, the complex64 Z (mixed precision) and / or separate B (Ne x Nv) and
// C (Nv x Nv) buffers (the refinement's exact operator); null pointers are skipped
struct BorderOut { double *Zd; float *Zf; long ld; double *B; double *C; };

__device__ __forceinline__ void put(const BorderOut &o, size_t zi, zd v)
{
    if (o.Zd) stc<double>(o.Zd, zi, v);
    if (o.Zf) stc<float>(o.Zf, zi, mk<float>((float)v.x, (float)v.y));
}

__global__ void k_via_B(const double *T, const double *c, int Nv, m25_mesh g, double w, BorderOut o)
{
    long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (idx >= (long)g.Ne * Nv) return;
    int e = idx / Nv, n = idx % Nv;
    const zd inv_jw = mk<double>(0, -1.0 / w);
    int p = g.ep[e], m = g.em[e];
    zd tp = ldc<double>(T, (size_t)p * Nv + n) * inv_jw + ldc<double>(c, (size_t)p * Nv + n);
    zd tm = ldc<double>(T, (size_t)m * Nv + n) * inv_jw + ldc<double>(c, (size_t)m * Nv + n);
    zd v = tp * (2 * g.ap[e]) + tm * (2 * g.am[e]);
    put(o, (size_t)e * o.ld + g.Ne + n, v);
    put(o, (size_t)(g.Ne + n) * o.ld + e, v);
    if (o.B) stc<double>(o.B, idx, v);
}

// C[m, n] = sum over chain m's fan entries (j, weight) weight T[F[j], n] / jw + R[m, n] into Z[Ne + m, Ne + n]
__global__ void k_via_C(const double *T, const int *F, const int *ptr, const int *fj, const double *fw, int Nv,
                        const double *Rm, int Ne, double w, BorderOut o)
{
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= Nv * Nv) return;
    int m = idx / Nv, n = idx % Nv;
    const zd inv_jw = mk<double>(0, -1.0 / w);
    zd acc = mk<double>(0, 0);
    for (int k = ptr[m]; k < ptr[m + 1]; ++k) acc += ldc<double>(T, (size_t)F[fj[k]] * Nv + n) * fw[k];
    zd v = acc * inv_jw + ldc<double>(Rm, idx);
    put(o, (size_t)(Ne + m) * o.ld + Ne + n, v);
    if (o.C) stc<double>(o.C, idx, v);
}

// R[m, n] (and R[n, m]) = vals[k] for the via pairs (m[k] <= n[k]); lerp from a table when tab != NULL
__global__ void k_via_pairs(const int *pm, const int *pn, const double *dd, int np, const double *vals,
                            const double *homog, const double *tab, long nfine, double dr, int Nv, double *R)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np) return;
    zd v;
    if (tab) {
        const double top = (double)nfine - 1.000001;
        double u = fmin(dd[k] / dr, top);
        long i = (long)u;
        double f = u - (double)i;
        v = ldc<double>(tab, i) * (1 - f) + ldc<double>(tab, i + 1) * f;
    } else {
        v = ldc<double>(vals, k);
    }
    v += ldc<double>(homog, k);
    int m = pm[k], n = pn[k];
    stc<double>(R, (size_t)m * Nv + n, ldc<double>(R, (size_t)m * Nv + n) + v);
    if (m != n) stc<double>(R, (size_t)n * Nv + m, ldc<double>(R, (size_t)n * Nv + m) + v);
}

extern "C" int m25_via_qcorr(double *d_QF, int nf, const int *d_pair, const int *d_row, const int *d_col, int n,
                             const double *d_qcorr, void *stream)
{
    if (!n) return M25_OK;
    k_qcorr_scatter<<<(n + 255) / 256, 256, 0, S(stream)>>>(d_QF, nf, d_pair, d_row, d_col, n, d_qcorr);
    M25_LAUNCH_CHECK("k_qcorr_scatter");
    return M25_OK;
}

extern "C" int m25_via_fan_T(const double *d_QF, int Nt, int nf, const int *d_ptr, const int *d_fj, const double *d_fw,
                             int Nv, double *d_T, void *stream)
{
    long tot = (long)Nt * Nv;
    if (!tot) return M25_OK;
    k_fan_T<<<(tot + 255) / 256, 256, 0, S(stream)>>>(d_QF, Nt, nf, d_ptr, d_fj, d_fw, Nv, d_T);
    M25_LAUNCH_CHECK("k_fan_T");
    return M25_OK;
}

extern "C" int m25_via_radial(const double *d_P6, const double *d_W6, const int *d_lt, int Nt, const double *d_vx,
                              const double *d_vy, const int *d_span_of, int Nv, const double *d_D, const int *d_dtab,
                              int nspan, long nfine, double dr, double *d_c, void *stream)
{
    long tot = (long)Nt * Nv;
    if (!tot) return M25_OK;
    k_radial_layers<<<(tot + 255) / 256, 256, 0, S(stream)>>>(d_P6, d_W6, d_lt, Nt, d_vx, d_vy, d_span_of, Nv, d_D,
                                                               d_dtab, nspan, nfine, dr, d_c);
    M25_LAUNCH_CHECK("k_radial_layers");
    return M25_OK;
}

extern "C" int m25_via_assemble(const double *d_T, const double *d_c, const int *d_F, const int *d_ptr,
                                const int *d_fj, const double *d_fw, int Nv, const double *d_R, const m25_mesh *g,
                                double w, double *d_Z, float *d_Z64, long ld, double *d_B, double *d_C, void *stream)
{
    M25_REQUIRE(g && ((!d_Z && !d_Z64) || ld >= g->Ne + Nv), "m25_via_assemble: mesh and ld >= Ne + Nv");
    if (!Nv) return M25_OK;
    BorderOut o{d_Z, d_Z64, ld, d_B, d_C};
    long tot = (long)g->Ne * Nv;
    k_via_B<<<(tot + 255) / 256, 256, 0, S(stream)>>>(d_T, d_c, Nv, *g, w, o);
    M25_LAUNCH_CHECK("k_via_B");
    k_via_C<<<(Nv * Nv + 255) / 256, 256, 0, S(stream)>>>(d_T, d_F, d_ptr, d_fj, d_fw, Nv, d_R, g->Ne, w, o);
    M25_LAUNCH_CHECK("k_via_C");
    return M25_OK;
}

extern "C" int m25_via_pairs(const int *d_pm, const int *d_pn, const double *d_dd, int np, const double *d_vals,
                             const double *d_homog, const double *d_tab, long nfine, double dr, int Nv, double *d_R,
                             void *stream)
{
    if (!np) return M25_OK;
    k_via_pairs<<<(np + 255) / 256, 256, 0, S(stream)>>>(d_pm, d_pn, d_dd, np, d_vals, d_homog, d_tab, nfine, dr, Nv,
                                                         d_R);
    M25_LAUNCH_CHECK("k_via_pairs");
    return M25_OK;
}
