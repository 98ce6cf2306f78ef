/*
 * mom25d_b200.h - the C ABI of libmom25d_b200.so: the per-frequency hot path of the 2.5-D MoM solver (Green
 * tables, impedance-matrix fill, near-field correction, via kernels, complex dense LU and solves) on one B200.
 *
 * Conventions
 *   - Every pointer named d_* is DEVICE memory; h_* is host memory. Matrices are row-major NumPy layouts
 *     (complex = interleaved re, im pairs of double or float). Z (N x N, row-major, leading dimension ld) is the
 *     reference's impedance matrix; its memory read column-major is Z^T, which the LU factors (as the reference's
 *     SciPy call does).
 *   - stream is a cudaStream_t passed as void* (0: the legacy default stream). Calls are asynchronous on it
 *     unless they say otherwise.
 *   - Every call returns M25_OK (0) or an error code; m25_last_error() gives the message of the calling thread's
 *     last error. Nothing here falls back to the CPU: no CUDA device or no kernel image is an error.
 *
 * Each entry point names the reference interface it replaces (lowprocess/mom25d, file:line).
 */
#ifndef MOM25D_B200_H
#define MOM25D_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define M25_OK 0
#define M25_EINVAL 1       /* bad argument (sizes, null pointers) */
#define M25_ECUDA 2        /* a CUDA runtime error (message in m25_last_error) */
#define M25_ENOMEM 3       /* workspace too small */
#define M25_EDEVICE 4      /* a kernel's own check failed: see the device code in m25_last_error */
#define M25_DEV_TIMEOUT 101   /* device codes: a bounded wait gave up */
#define M25_DEV_INDEX 102     /*               an index out of range was skipped */
#define M25_DEV_ZEROPIV 103   /*               an exactly zero pivot (the factor is singular) */

/* The packed mesh (mom25d fast.py:391-396, the compiled core's `g`): Ne edges, Nt triangles; device pointers.
 * ep, em int32[Ne]; lt int32[Nt] (interface index into the table map); te int32[Nt*3]; ap, am f64[Ne];
 * vp, vm f64[Ne*2]; cent f64[Nt*2]; area f64[Nt]; ta f64[Nt*3]; tv f64[Nt*6]. */
typedef struct m25_mesh {
    int Ne, Nt;
    const int *ep, *em, *lt, *te;
    const double *ap, *am, *vp, *vm, *cent, *area, *ta, *tv;
} m25_mesh;

/* The Green tables (fast.py:556-568, the compiled core's `tb`): ntab tables of nfine uniform samples from rho = 0
 * step dr[t]; A, Q complex128[ntab*nfine]; cA, cq, cAi, cqi complex128[ntab] (singular coefficients); d, dimg
 * f64[ntab]; tab int32[L*L] (table of an interface pair); kind int32[ntab] (0 same interface, 1 cross with the
 * near-singular part extracted, 2 cross plain). */
typedef struct m25_tables {
    int ntab, nfine, L;
    const double *A, *Q, *cA, *cq, *cAi, *cqi;
    const double *dr, *d, *dimg;
    const int *tab, *kind;
} m25_tables;

/* The same tables in single precision for the mixed-precision fill (complex64 samples and coefficients). */
typedef struct m25_tables_f {
    int ntab, nfine, L;
    const float *A, *Q, *cA, *cq, *cAi, *cqi;
    const float *dr, *d, *dimg;
    const int *tab, *kind;
} m25_tables_f;

/* Quadrature and vertex data of the near-field correction (fast.py:397-398, the core's `q`): nodes f64[Nn*2],
 * tris int32[Nt*3], P3 f64[Nt*3*2], W3 f64[Nt*3], P6 f64[Nt*6*2], W6 f64[Nt*6]. */
typedef struct m25_quad {
    const double *nodes;
    const int *tris;
    const double *P3, *W3, *P6, *W6;
} m25_quad;

const char *m25_version(void);
const char *m25_last_error(void);
/* SM count, free and total device memory of the current device (replaces gpu.py:28-48 mem_free / mem_total). */
int m25_device_info(int *sm_count, size_t *free_bytes, size_t *total_bytes);

/* ---- Green tables (multilayer.py:183-318, via.py:36-123) ------------------------------------------------------ */
/* Spectral kernels of the stack's transmission-line network at npts points kr of the Sommerfeld contour, for
 * npair interface pairs (o[i], s[i]) (multilayer.py:183-250 _network / voltage / spectral). Layers: nl layers of
 * thickness h[j] and complex permittivity eps[2j], eps[2j+1]; top_open != 0: a half-space of top_eps above, else a
 * PEC cover. Writes GA, GQ complex128[npair*npts] (pair-major). mode_tm_only != 0: write the TM voltage V_e in
 * GA and leave GQ alone (the via kernels' network, via.py:127-166). */
int m25_spectral(const double *d_kr, int npts, double w, int nl, const double *h_h, const double *h_eps,
                 int top_open, const double *h_top_eps, int npair, const int *h_o, const int *h_s,
                 double *d_GA, double *d_GQ, void *stream);
/* out[s, i] = (1/2pi) sum_k J0(rho_i kr_k) W[s, k] kr_k dk_k over a contour whose first nlift points are complex
 * (replaces via.py:104-108 hankel, with mom25d_core.cpp:1430-1454 hankel_real and :1510-1558 bessel_jn_complex).
 * kr, dk complex128[npts]; W complex128[ns*npts]; rho f64[nr]; out complex128[ns*nr]. */
int m25_hankel(const double *d_kr, const double *d_dk, int npts, const double *d_W, int ns, const double *d_rho,
               int nr, double *d_out, void *stream);
/* out[s, i] = sum_k J0(rho_i kr_k) W[s, k] over real kr f64[nk] (hankel_real, mom25d_core.cpp:1430-1454);
 * W complex128[ns*nk], out complex128[ns*nr], ns <= 16. */
int m25_hankel_real(const double *d_rho, int nr, const double *d_kr, int nk, const double *d_W, int ns,
                    double *d_out, void *stream);
/* Not-a-knot cubic spline through (x[i], y[s, i]), i < n, evaluated at nfine uniform points from 0 step dx
 * (via.py:111-123 Table1D, SciPy CubicSpline). y complex128[ns*n]; out: complex128 or (single) complex64
 * [ns*nfine]; out_stride: elements between rows. */
int m25_spline_uniform(const double *d_x, const double *d_y, int ns, int n, double dx, int nfine, void *d_out,
                       int single, long out_stride, long out_offset_elems, int out_interleave, void *stream);
/* The spectral kernels of npair (<= 64) interface pairs with their singular parts subtracted in the spectral
 * domain before the Hankel transform (GreenTableML.__init__ / extracted, multilayer.py:260-299): per pair i,
 * next[i] (0..2) extracted terms of distance d[2i + j] and coefficients cA, cq (complex128, host [npair*2]).
 * d_pairs_scratch: m25_pair_record_bytes() device bytes. Synchronous in its host-to-device copy of the records. */
int m25_spectral_extracted(const double *d_kr, int npts, double w, int nl, const double *h_h, const double *h_eps,
                           int top_open, const double *h_top_eps, int npair, const int *h_o, const int *h_s,
                           const int *h_next, const double *h_d, const double *h_cA, const double *h_cq,
                           double *d_GA, double *d_GQ, void *d_pairs_scratch, void *stream);
size_t m25_pair_record_bytes(void);
/* The spectral kernels G_A, G_q of one interface pair (o, s) at npts (kr, w) points, each point its own angular
 * frequency w[i] (real): the large-kr limits that give the extraction coefficients (multilayer.py:271-287). */
int m25_spectral_points(const double *d_kr, const double *d_w, int npts, int nl, const double *h_h,
                        const double *h_eps, int top_open, const double *h_top_eps, int o, int s, double *d_ga,
                        double *d_gq, void *stream);

/* ---- via kernels (via.py:127-235 TMNetwork / ViaKernels, sim.py:786-872 _via_blocks) --------------------------- */
/* The via spectra on the contour: nd (<= 32) D spectra (strip interface dk[i], via span dspan[2i..2i+1]) then
 * nr (<= 32) R spectra (span rm[2i..] against span rn[2i..], without the homogeneous term) (via.py:205-220);
 * out complex128[(nd + nr) * npts], row-major by spectrum. */
int m25_via_spectra(const double *d_kr, int npts, double w, int nl, const double *h_h, const double *h_eps,
                    int top_open, const double *h_top_eps, int nd, const int *h_dk, const int *h_dspan, int nr,
                    const int *h_rm, const int *h_rn, double *d_out, void *stream);
/* The analytic homogeneous (K0) term of the via-via kernel at n distances rho for the layers in layer_mask
 * (via.py:222-235 ViaKernels.homog); out complex128[n]. */
int m25_via_homog(const double *d_rho, int n, double w, int nl, const double *h_h, const double *h_eps,
                  int top_open, const double *h_top_eps, unsigned layer_mask, double *d_out, void *stream);
/* QF[row[k], col[k]] += qcorr[pair[k]]: the near pairs' G_q corrections on the fan columns (fast.py:501-503).
 * QF complex128[Nt*nf]. */
int m25_via_qcorr(double *d_QF, int nf, const int *d_pair, const int *d_row, const int *d_col, int n,
                  const double *d_qcorr, void *stream);
/* T[t, n] = sum over chain n's fan entries (fj[k], fw[k]), k in ptr[n]..ptr[n+1], of QF[t, fj[k]] fw[k]
 * (the fan charges dF of sim.py:840-849); T complex128[Nt*Nv]. */
int m25_via_fan_T(const double *d_QF, int Nt, int nf, const int *d_ptr, const int *d_fj, const double *d_fw, int Nv,
                  double *d_T, void *stream);
/* c[t, n] = sum over the 6 points of triangle t of D(|P6 - V_n|) W6, D the table dtab[lt[t] * nspan + span_of[n]]
 * of D complex128[ntables*nfine] (radial_table_sum per interface and span, mom25d_core.cpp:1269-1298). */
int m25_via_radial(const double *d_P6, const double *d_W6, const int *d_lt, int Nt, const double *d_vx,
                   const double *d_vy, const int *d_span_of, int Nv, const double *d_D, const int *d_dtab, int nspan,
                   long nfine, double dr, double *d_c, void *stream);
/* The via border: B = D^T (T / jw + c) (Ne x Nv) and C = dF^T T / jw + R (Nv x Nv) (sim.py:850-872), written into
 * the bordered Z (complex128 d_Z and / or complex64 d_Z64, leading dimension ld >= Ne + Nv: columns and rows
 * Ne..Ne+Nv-1) and / or separate d_B, d_C buffers; null destinations are skipped. */
int m25_via_assemble(const double *d_T, const double *d_c, const int *d_F, const int *d_ptr, const int *d_fj,
                     const double *d_fw, int Nv, const double *d_R, const m25_mesh *g, double w, double *d_Z,
                     float *d_Z64, long ld, double *d_B, double *d_C, void *stream);
/* R[m, n] += vals[k] (or the lerp of tab at dd[k] when d_tab != NULL) + homog[k], and R[n, m] the same, for the
 * np via pairs (pm[k] <= pn[k]) (the via-via R kernel, via.py:188-221); R complex128[Nv*Nv]. */
int m25_via_pairs(const int *d_pm, const int *d_pn, const double *d_dd, int np, const double *d_vals,
                  const double *d_homog, const double *d_tab, long nfine, double dr, int Nv, double *d_R,
                  void *stream);

/* ---- fill (mom25d_core.cpp) ------------------------------------------------------------------------------------ */
/* Centroid-rule far field of every edge pair into Z (Ne x Ne block of a row-major N x ld matrix), both
 * triangles written (fill_far / fill_far_c64, mom25d_core.cpp:132-173). single: Z complex64 from the complex64
 * tables tbf (the mixed-precision fill), else complex128 from tb. */
int m25_fill_far(void *d_Z, long ld, int single, const m25_mesh *g, const m25_tables *tb, const m25_tables_f *tbf,
                 double w, void *stream);
/* The far fill of several frequencies of one board in one launch (the reference fills one frequency a call,
 * fill_far, mom25d_core.cpp:132-173; this serves a batched sweep): d_Zs a device array of nf matrix pointers
 * (row-major N x ld each, complex128 or complex64 by `single`), d_tables a device array of nf m25_tables
 * (complex128) or m25_tables_f (complex64) structs, d_w the nf angular frequencies on the device. Each Z gets
 * exactly what m25_fill_far writes for its frequency. */
int m25_fill_far_multi(void *const *d_Zs, long ld, int single, const m25_mesh *g, const void *d_tables,
                       const double *d_w, int nf, void *stream);
/* The far field for row / column edge lists: out complex128[nr*nc] (far_block, mom25d_core.cpp:176-211). */
int m25_far_block(const int *d_rows, int nr, const int *d_cols, int nc, double *d_out, const m25_mesh *g,
                  const m25_tables *tb, double w, void *stream);
/* Near-field correction of n near triangle pairs (P[i], Q[i]) (near_core, mom25d_core.cpp:417-507).
 * mode 0: added into Z (complex128, or complex64 if single) (near_into_dense :520);
 * mode 2: COO triplets ri, ci int32[9n] (-1 unused), vv complex128[9n] (near_coo :559);
 * qcorr complex128[n] (may be null) gets each pair's G_q moment correction. stat f64[12n] keeps the pairs'
 * analytic parts across frequencies: stat_ready = 0 computes and stores them, 1 reads them. */
int m25_near(int mode, void *d_Z, long ld, int single, int *d_ri, int *d_ci, double *d_vv, double *d_qcorr,
             double *d_stat, int stat_ready, const m25_mesh *g, const m25_tables *tb, const m25_quad *q,
             const int *d_P, const int *d_Q, long n, double w, void *stream);
/* Near triangle pairs: rho^2 + dz^2 < (fac max(size_p, size_q))^2, sorted by (p, q) (near_pairs,
 * mom25d_core.cpp:1216-1263). Two calls: d_P == NULL writes the per-row counts into d_offsets (int64[Nt+1], an
 * exclusive scan) and *h_total; then d_P, d_Q (int32[total]) are filled. Synchronous. */
int m25_near_pairs(const double *d_cent, const double *d_size, const double *d_z, int Nt, double fac,
                   long long *d_offsets, long long *h_total, int *d_P, int *d_Q, void *stream);
/* G_q x area_t x area_f between every triangle t and the fan triangles F[j]: out complex128[Nt*nf]
 * (fan_q, mom25d_core.cpp:1585-1603). */
int m25_fan_q(const int *d_F, int nf, double *d_out, const m25_mesh *g, const m25_tables *tb, void *stream);
/* out[t, v] = sum_q D(|P[t, q] - V[v]|) W[t, q] for a radial table D complex128[n] of step dr
 * (radial_table_sum, mom25d_core.cpp:1269-1298); px, py, W f64[nt*nq]; vx, vy f64[nv]; out complex128[nt*nv]. */
int m25_radial_table_sum(const double *d_px, const double *d_py, const double *d_W, long nt, int nq,
                         const double *d_vx, const double *d_vy, int nv, const double *d_table, long n, double dr,
                         double *d_out, void *stream);
/* Y = Z_far X for K columns without Z (matvec_far_multi, mom25d_core.cpp:257-314); X, Y complex128[Ne*K];
 * work: 6*Nt*K complex128. */
int m25_matvec_far_multi(const double *d_X, int K, double *d_Y, double *d_work, const m25_mesh *g,
                         const m25_tables *tb, double w, void *stream);
/* Z <- diag(d) Z diag(d) in place, and (if d_Z64 != NULL) its complex64 copy (scale_c64,
 * mom25d_core.cpp:1563-1580; _equilibrate fast.py:294-305). dsc: if d_dsc_out != NULL, first computes
 * d = 1 / sqrt(|Z_ii| + 1e-300) into it and uses that. */
int m25_equilibrate(double *d_Z, long n, long ld, const double *d_d, double *d_dsc_out, float *d_Z64, void *stream);
/* The same for a complex64 Z (the mixed-precision fill writes complex64 directly): d from its diagonal into
 * d_dsc_out (f64[n]), Z <- diag(d) Z diag(d). */
int m25_equilibrate_c64(float *d_Z, long n, long ld, double *d_dsc_out, void *stream);

/* ---- the exact FP64 operator and the refinement's vector kernels (fast.py:571-593, 1437-1500) ----------------- */
/* Vectors are N x k row-major complex128 (one column per right-hand side). */
/* out[c] += sum_n conj(V[n, c]) W[n, c] (out zeroed by the caller). */
int m25_dotc_cols(const double *d_V, const double *d_W, long N, int k, double *d_out, void *stream);
/* W[n, c] += V[n, c] a[c]. */
int m25_axpy_cols(double *d_W, const double *d_V, const double *d_a, long N, int k, void *stream);
/* The Gram-Schmidt step against a whole Krylov basis (batched GMRES, fast.py:1437-1500, as classical Gram-Schmidt
 * applied twice): out[i, c] = sum_n conj(V_i[n, c]) W[n, c] for the nv blocks V_i (N x k each, consecutive);
 * W -= sum_i V_i h[i, c] (h complex128[nv * k]). */
int m25_dotc_multi(const double *d_V, int nv, long N, int k, const double *d_W, double *d_out, void *stream);
int m25_axpy_multi(double *d_W, const double *d_V, int nv, long N, int k, const double *d_h, void *stream);
/* One Arnoldi step of the batched GMRES (replaces the per-vector modified Gram-Schmidt loop of gmres_batched,
 * fast.py:1470-1476) without a host round trip: W orthogonalised against the basis blocks V_0 .. V_j (classical
 * Gram-Schmidt applied twice) and normalised into V_{j+1} = d_V + (j + 1) N k complex; the Hessenberg column
 * (j + 1 projections, then the norm as a real) into d_h ((j + 2) x k complex128). d_tmp: (j + 1) x k complex128. */
int m25_arnoldi_orth(double *d_V, int j, long N, int k, double *d_W, double *d_h, double *d_tmp, void *stream);
/* Y[n, c] = X[n, c] s[c] (times rows[n] when d_rows != NULL); s complex128[k] or NULL for 1. */
int m25_scale_cols(double *d_Y, const double *d_X, const double *d_s, const double *d_rows, long N, int k,
                   void *stream);
/* n complex numbers complex128 -> complex64 (in_single = 0) or complex64 -> complex128 (in_single = 1). */
int m25_convert(const void *d_in, int in_single, void *d_out, long n, void *stream);
/* Y[ri[s], c] += vv[s] X[ci[s], c] over COO triplets (ri < 0 unused; near_matvec, mom25d_core.cpp:540-556). */
int m25_coo_spmm(const int *d_ri, const int *d_ci, const double *d_vv, long nnz, const double *d_X, int k,
                 double *d_Y, void *stream);
/* The same product row by row without atomics (deterministic): the triplets of m25_near mode 2 in pair order,
 * off int64[Nt+1] the pairs of each observation triangle, Q the source triangles. */
int m25_near_spmm_rows(const m25_mesh *g, const long long *d_off, const int *d_Q, const double *d_vv,
                       const double *d_X, int k, double *d_Y, void *stream);
/* Z (complex64, ld) += vv at (ri, ci): the near field into the mixed-precision matrix. */
int m25_coo_add_c64(const int *d_ri, const int *d_ci, const double *d_vv, long nnz, float *d_Z, long ld,
                    void *stream);
/* Z (row-major n x n, leading dimension ld; complex64 when single, else complex128) += vv (complex128) at the
 * distinct entries (ri, ci): the lumped elements and conductor loss of the reference's extra_blocks
 * (fast.py:628-641), added into the filled Z. An index outside [0, n) is reported by m25_sync_check. */
int m25_coo_add(const int *d_ri, const int *d_ci, const double *d_vv, long nnz, void *d_Z, long ld, int n, int single,
                void *stream);
/* Y = Z X for a resident double Z (row-major n x n, leading dimension ld) and X (n x k, k <= 16): the dense
 * products of the refinement when the double Z stays on the device (fast.py:1009, _solve_kept: A = Z @ V). */
int m25_zgemm_skinny(const double *d_Z, long ld, int n, const double *d_X, int k, double *d_Y, void *stream);
/* The via border of Z X (fast.py:580-586): Y[:Ne] += B X[Ne:], Y[Ne:] = B^T X[:Ne] + C X[Ne:]. */
int m25_border_mv(const double *d_B, const double *d_C, int Ne, int Nv, const double *d_X, int k, double *d_Y,
                  void *stream);

/* ---- complex dense LU (gpu.py:28-110 backend factor / solve / download; fast.py:318-358 _lu / _lu_solve) ------- */
/* Workspace bytes m25_getrf needs for an n x n factorisation. */
size_t m25_getrf_workspace(int n, int single);
/* LU with partial pivoting of A = Z^T in place (A column-major n x n, leading dimension lda: the memory of the
 * row-major Z), LAPACK's zgetrf / cgetrf semantics: A = P L U, L unit lower; ipiv int32[n] 0-based (row i was
 * interchanged with row ipiv[i]), like scipy.linalg.lu_factor. single: complex64, else complex128. tf32 (single
 * only): trailing updates on the tensor cores as 3xTF32 products. */
int m25_getrf(void *d_A, long lda, int n, int *d_ipiv, int single, int tf32, void *d_work, size_t work_bytes,
              void *stream);
/* The LU's tile parameters by matrix size (no counterpart in the reference: LAPACK picks its own blocking): a
 * table for complex64 (single = 1) and one for complex128 factorisations, up to 32 entries each (n, outer panel
 * width nb2 = 64..256 in steps of 64, cooperative panel blocks), as the autotuner (mom25d_b200/tune.py) finds them
 * on this GPU; a factorisation of size n takes the entry nearest to n in log n. count 0 restores the defaults
 * (256, min(SMs, 32)). The environment variables M25_NB2 and M25_PANEL_BLOCKS override both.
 * m25_get_lu_tuning: what a factorisation of size n uses. */
int m25_set_lu_tuning(int single, const int *h_n, const int *h_nb2, const int *h_blocks, int count);
int m25_get_lu_tuning(int n, int single, int *nb2, int *blocks);
/* Solves Z X = B with the factor of Z^T (lu_solve(..., trans=1)); B (row-major n x nrhs, complex in the factor's
 * precision) overwritten by X. One call: its scratch from the stream-ordered allocator, by 64-row diagonal blocks
 * (for many solves with one factor, m25_getrs_prepare / m25_getrs_aux below). */
int m25_getrs(const void *d_LU, long lda, int n, const int *d_ipiv, int single, void *d_B, int nrhs, void *stream);
/* The solves split for a factor that is solved with many times (the refinement's preconditioner, the backend's
 * solve(R)): m25_getrs_prepare inverts the factor's diagonal blocks once into d_aux (m25_getrs_aux_bytes) and
 * keeps the pivots there; m25_getrs_aux then solves like m25_getrs from d_aux. d_aux belongs to one factor, and its
 * solves run one at a time (they share its flags and work vectors: two on different streams race). For a
 * factor of n >= 2048, d_aux also holds the inverses of its 256-row diagonal blocks and their couplings with the
 * two blocks before them (three 256 x 256 matrices a block a triangle), with which solves of up to 8 right-hand
 * sides take one product a block along their chain (M25_TRSV=pipe: not; M25_TRSV=c64: complex64 factors only). */
size_t m25_getrs_aux_bytes(int n, int single);
int m25_getrs_prepare(const void *d_LU, long lda, int n, const int *d_ipiv, int single, void *d_aux,
                      size_t aux_bytes, void *stream);
int m25_getrs_aux(const void *d_LU, long lda, int n, int single, void *d_aux, void *d_B, int nrhs, void *stream);
/* m25_getrs without device allocation (no counterpart in the reference). m25_getrs takes its scratch from the
 * stream-ordered allocator at every call; this variant uses a fixed file-scope device array of
 * M25_GETRS_NOALLOC_MAX_BYTES instead, for callers that must not have the library take device memory during a
 * call: a serving loop that admits requests by a fixed HBM budget, or a process whose memory is all reserved up
 * front. Same arguments as m25_getrs and its results to rounding (it always solves by 64-row diagonal blocks).
 * Limit: n whose data for those solves
 * (inverses, permutation, work vectors, flags) is above M25_GETRS_NOALLOC_MAX_BYTES (about n = 26,000 complex64,
 * 13,000 complex128) is rejected with M25_EINVAL and a
 * message. The first call on a device does the setup (it looks up the array's device address); make it before
 * any stream capture. The array is one per device and process: calls that overlap (other streams, other host
 * threads on the same device) race on it and must be serialised by the caller. A bounded wait that gave up is
 * reported by m25_sync_check, as for the other kernels. */
#define M25_GETRS_NOALLOC_MAX_BYTES (32u << 20)
int m25_getrs_noalloc(const void *d_LU, long lda, int n, const int *d_ipiv, int single, void *d_B, int nrhs,
                      void *stream);
/* The LU's tensor-core trailing update alone: C (M x N complex64, column-major, ld) -= L (M x K) U (K x N), both
 * column-major with leading dimension ld, as 3xTF32 products on tcgen05. work: split operands. */
int m25_cgemm_update_tf32(float *d_C, long ld, int M, int N, int K, const float *d_L, const float *d_U, void *d_work,
                          size_t work_bytes, void *stream);
/* 1 when the library carries the tensor-core (tcgen05) update. */
int m25_umma_available(void);
/* The tensor-core update's work split (no counterpart in the reference): `tiles` = 1 gives one output tile a CTA,
 * two CTAs an SM; more gives runs of that many consecutive tiles a CTA, one CTA an SM, with two tensor-memory
 * accumulators so each tile's epilogue runs under the next tile's MMAs - for updates of at least min_tiles tiles
 * (min_tiles < 0: two an SM). M25_UMMA_TPC in the environment overrides `tiles`. */
int m25_set_umma_tiles(int tiles, int min_tiles);

/* ---- small helpers ------------------------------------------------------------------------------------------------ */
/* J_n(z) elementwise for complex z, n = 0, 1, 2 (bessel_jn_complex, mom25d_core.cpp:1545-1558). */
int m25_bessel_jn_complex(int order, const double *d_z, long count, double *d_out, void *stream);
/* Synchronises stream and turns a pending kernel error (or a device-side check, M25_EDEVICE) into a status. */
int m25_sync_check(void *stream);
/* Exercises the failure-detection path (no counterpart in the reference, whose CPU and Vulkan paths have no device
 * waits): the cooperative kernels' bounded grid barrier entered by one block that waits for a block never
 * launched. The wait gives up at its iteration limit (a few seconds), the kernel returns, and the next
 * m25_sync_check reports M25_EDEVICE (M25_DEV_TIMEOUT) with the context still usable. */
int m25_wait_selftest(void *stream);
/* How many kernels this library has launched in the process (a counter for measurements). */
long long m25_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif
