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
/* Not-a-knot cubic spline through (x[i], y[s, i]), i < n, evaluated at nfine uniform points from 0 step dx
 * (via.py:111-123 Table1D, SciPy CubicSpline). y complex128[ns*n]; out: complex128 or (single) complex64
 * [ns*nfine]; out_stride: elements between rows. */
int m25_spline_uniform(const double *d_x, const double *d_y, int ns, int n, double dx, int nfine, void *d_out,
                       int single, long out_stride, long out_offset_elems, int out_interleave, void *stream);

/* ---- fill (mom25d_core.cpp) ------------------------------------------------------------------------------------ */
/* Centroid-rule far field of every edge pair into Z (Ne x Ne block of a row-major N x ld matrix), both
 * triangles written (fill_far / fill_far_c64, mom25d_core.cpp:132-173). single: Z complex64 from the complex64
 * tables tbf (the mixed-precision fill), else complex128 from tb. */
int m25_fill_far(void *d_Z, long ld, int single, const m25_mesh *g, const m25_tables *tb, const m25_tables_f *tbf,
                 double w, void *stream);
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

/* ---- complex dense LU (gpu.py:28-110 backend factor / solve / download; fast.py:318-358 _lu / _lu_solve) ------- */
/* Workspace bytes m25_getrf needs for an n x n factorisation. */
size_t m25_getrf_workspace(int n, int single);
/* LU with partial pivoting of A = Z^T in place (A column-major n x n, leading dimension lda: the memory of the
 * row-major Z), LAPACK's zgetrf / cgetrf semantics: A = P L U, L unit lower; ipiv int32[n] 0-based (row i was
 * interchanged with row ipiv[i]), like scipy.linalg.lu_factor. single: complex64, else complex128. tf32 (single
 * only): trailing updates on the tensor cores as 3xTF32 products. */
int m25_getrf(void *d_A, long lda, int n, int *d_ipiv, int single, int tf32, void *d_work, size_t work_bytes,
              void *stream);
/* Solves Z X = B with the factor of Z^T (lu_solve(..., trans=1)); B (row-major n x nrhs, complex in the factor's
 * precision) overwritten by X. */
int m25_getrs(const void *d_LU, long lda, int n, const int *d_ipiv, int single, void *d_B, int nrhs, void *stream);

/* ---- small helpers ------------------------------------------------------------------------------------------------ */
/* J_n(z) elementwise for complex z, n = 0, 1, 2 (bessel_jn_complex, mom25d_core.cpp:1545-1558). */
int m25_bessel_jn_complex(int order, const double *d_z, long count, double *d_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
