// lu.cu - complex dense LU with partial pivoting (blocked, right-looking) and the triangular solves, on one GPU.
//
// The matrix is A = Z^T in column-major order: the memory of the reference's row-major impedance matrix Z, which
// LAPACK factors through SciPy (mom25d fast.py:318-320 _lu, lu_factor(Z.T)) and solves with trans = 1
// (fast.py:356-358). Pivots follow zgetrf: the largest |re| + |im| of the column (izamax), the first on ties.
//
// Per panel of nb columns:
//   1. k_panel     cooperative kernel over all SMs: the panel's rows split between the blocks; per column one grid
//                  barrier (bounded) after each block publishes its candidate pivot row, then every block applies
//                  the interchange and the rank-1 update to its own rows.
//   2. k_laswp     the panel's interchanges applied to the columns left and right of it.
//   3. k_trsm      U12 = L11^-1 A12 (unit lower), one thread per column, L11 in shared memory.
//   4. trailing    A22 -= L21 U12: the complex SIMT GEMM below (FP64 / FP32), or the tensor-core 3xTF32 product
//                  (umma.cu) for complex64 with tf32 on.
#include <cooperative_groups.h>
#include "common.cuh"

static inline cudaStream_t S(void *s) { return (cudaStream_t)s; }
int *m25_dev_err_word();
int m25_check_dev_err(cudaStream_t s, const char *what);
int m25_umma_trailing(float *A, long lda, int M, int Ncol, int K, const float *L21, const float *U12, void *work,
                      size_t work_bytes, cudaStream_t s);
size_t m25_umma_workspace(int n, int nb);

#define NB 64
#define PANEL_THREADS 256

struct PanelWork {
    double *cand_val;     // [2][G]
    int *cand_idx;        // [2][G]
    double *cand_row;     // [2][G][NB] complex (as R pairs; sized for double)
    double *drow;         // [2][NB] complex
    GridBarrier bar;
};

template <typename R>
__global__ void __launch_bounds__(PANEL_THREADS) k_panel(R *A, long lda, int n, int k0, int jb, int *ipiv, PanelWork pw,
                                                         int *err)
{
    typedef cpx<R> C;
    const unsigned G = gridDim.x;
    const int b = blockIdx.x, tid = threadIdx.x;
    const int rows = n - k0;
    const int cs = (rows + G - 1) / G;
    const int r0 = k0 + b * cs, r1 = min(n, r0 + cs);
    unsigned phase = 0;
    __shared__ C U[NB], D[NB];
    __shared__ double sv[PANEL_THREADS / 32];
    __shared__ int si[PANEL_THREADS / 32];
    __shared__ int s_p;
    __shared__ C s_recip;
    C *cand_row = reinterpret_cast<C *>(pw.cand_row);
    C *drow = reinterpret_cast<C *>(pw.drow);
    for (int j = 0; j < jb; ++j) {
        const int col = k0 + j, par = j & 1;
        // 1. local candidate: the largest |re| + |im| in column col among own rows >= col (the first on ties)
        double best = -1.0;
        int bi = 0x7fffffff;
        for (int r = max(r0, col) + tid; r < r1; r += PANEL_THREADS) {
            double v = abs1(ldc<R>(A, (size_t)col * lda + r));
            if (v > best) { best = v; bi = r; }
        }
        for (int o = 16; o; o >>= 1) {
            double ov = __shfl_xor_sync(0xffffffffu, best, o);
            int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        if ((tid & 31) == 0) { sv[tid >> 5] = best; si[tid >> 5] = bi; }
        __syncthreads();
        if (tid == 0) {
            for (int w = 1; w < PANEL_THREADS / 32; ++w)
                if (sv[w] > best || (sv[w] == best && si[w] < bi)) { best = sv[w]; bi = si[w]; }
            pw.cand_val[par * G + b] = best;
            pw.cand_idx[par * G + b] = bi;
            s_p = bi;
        }
        __syncthreads();
        if (s_p != 0x7fffffff && tid < jb)
            cand_row[((size_t)par * G + b) * NB + tid] = ldc<R>(A, (size_t)(k0 + tid) * lda + s_p);
        if (col >= r0 && col < r1 && tid < jb) drow[par * NB + tid] = ldc<R>(A, (size_t)(k0 + tid) * lda + col);
        // 2. all blocks' candidates published
        if (!grid_sync(pw.bar, G, phase, err)) return;
        // 3. the pivot: the best candidate over the blocks, the smallest row on ties
        if (tid == 0) {
            double bv = -1.0;
            int bw = -1, brow = 0x7fffffff;
            for (unsigned w = 0; w < G; ++w) {
                double v = ((volatile double *)pw.cand_val)[par * G + w];
                int ri = ((volatile int *)pw.cand_idx)[par * G + w];
                if (ri == 0x7fffffff) continue;
                if (v > bv || (v == bv && ri < brow)) { bv = v; bw = (int)w; brow = ri; }
            }
            si[0] = bw;
            s_p = brow;
            if (b == 0) ipiv[col] = brow;
        }
        __syncthreads();
        const int wb = si[0], p = s_p;
        if (wb < 0) { dev_error(err, M25_DEV_INDEX); return; }
        if (tid < jb) {           // other blocks' writes: read past L1
            const volatile R *cu = (const volatile R *)(cand_row + ((size_t)par * G + wb) * NB + tid);
            const volatile R *cd = (const volatile R *)(drow + par * NB + tid);
            U[tid] = mk<R>(cu[0], cu[1]);
            D[tid] = mk<R>(cd[0], cd[1]);
        }
        __syncthreads();
        // 4. the interchange, by the owners of the two rows
        if (tid < jb) {
            if (col >= r0 && col < r1) stc<R>(A, (size_t)(k0 + tid) * lda + col, U[tid]);
            if (p != col && p >= r0 && p < r1) stc<R>(A, (size_t)(k0 + tid) * lda + p, D[tid]);
        }
        if (tid == 0) {
            C piv = U[j];
            if (piv.x == 0 && piv.y == 0) { dev_error(err, M25_DEV_ZEROPIV); s_recip = mk<R>(0, 0); }
            else s_recip = cdiv<R>(mk<R>(1, 0), piv);
        }
        __syncthreads();
        // 5. scale the column below the diagonal and update the rest of the panel on own rows
        const C rc = s_recip;
        for (int r = max(r0, col + 1) + tid; r < r1; r += PANEL_THREADS) {
            C l = ldc<R>(A, (size_t)col * lda + r) * rc;
            stc<R>(A, (size_t)col * lda + r, l);
            for (int c = j + 1; c < jb; ++c) {
                C a = ldc<R>(A, (size_t)(k0 + c) * lda + r);
                cfms<R>(a, l, U[c]);
                stc<R>(A, (size_t)(k0 + c) * lda + r, a);
            }
        }
        __syncthreads();
    }
}

// the panel's interchanges on the columns outside it: one thread per column, the swaps in order
template <typename R>
__global__ void k_laswp(R *A, long lda, int n, int k0, int jb, const int *ipiv)
{
    long c = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (c >= n - jb) return;
    if (c >= k0) c += jb;                                  // skip the panel's own columns
    R *col = A + 2 * (size_t)c * lda;
    for (int j = 0; j < jb; ++j) {
        int p = ipiv[k0 + j], r = k0 + j;
        if (p != r && p >= 0 && p < n) {
            cpx<R> a = ldc<R>(col, r), b = ldc<R>(col, p);
            stc<R>(col, r, b); stc<R>(col, p, a);
        }
    }
}

// U12 = L11^-1 A12: L11 (jb x jb, unit lower) in shared memory, each thread one column of A12
template <typename R>
__global__ void __launch_bounds__(64) k_trsm(R *A, long lda, int n, int k0, int jb)
{
    typedef cpx<R> C;
    extern __shared__ unsigned char sm_raw[];
    C *L = reinterpret_cast<C *>(sm_raw);                  // L[i * NB + k]
    C *X = L + NB * NB;                                    // X[i * 64 + thread]
    for (int e = threadIdx.x; e < jb * jb; e += blockDim.x) {
        int k = e / jb, i = e % jb;                        // column k, row i (column-major read, coalesced)
        L[i * NB + k] = ldc<R>(A, (size_t)(k0 + k) * lda + k0 + i);
    }
    const long c = k0 + jb + blockIdx.x * (long)blockDim.x + threadIdx.x;
    const bool live = c < n;
    if (live)
        for (int i = 0; i < jb; ++i) X[i * 64 + threadIdx.x] = ldc<R>(A, (size_t)c * lda + k0 + i);
    __syncthreads();
    if (!live) return;
    for (int i = 1; i < jb; ++i) {
        C x = X[i * 64 + threadIdx.x];
        for (int k = 0; k < i; ++k) cfms<R>(x, L[i * NB + k], X[k * 64 + threadIdx.x]);
        X[i * 64 + threadIdx.x] = x;
    }
    for (int i = 0; i < jb; ++i) stc<R>(A, (size_t)c * lda + k0 + i, X[i * 64 + threadIdx.x]);
}

// C (M x N) -= A (M x K) B (K x N), all column-major complex inside the factor (lda). 128 x 64 tile per block of
// 256 threads, each 8 x 4 outputs; K staged 16 at a time through shared memory (the next slice prefetched into
// registers while the current one is used).
template <typename R>
__global__ void __launch_bounds__(256) k_gemm_update(R *Cm, const R *Am, const R *Bm, long lda, int M, int N, int K)
{
    typedef cpx<R> C;
    constexpr int BM = 128, BN = 64, BK = 8;
    __shared__ C As[BK][BM];
    __shared__ C Bs[BK][BN + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    C acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = mk<R>(0, 0);
    for (int kk = 0; kk < K; kk += BK) {
        // A slice: BK columns of BM rows (coalesced along rows)
        for (int e = threadIdx.x; e < BK * BM; e += 256) {
            int k = e / BM, m = e % BM;
            As[k][m] = (m0 + m < M && kk + k < K) ? ldc<R>(Am, (size_t)(kk + k) * lda + m0 + m) : mk<R>(0, 0);
        }
        // B slice: BN columns of BK rows (coalesced along k)
        for (int e = threadIdx.x; e < BK * BN; e += 256) {
            int nn = e / BK, k = e % BK;
            Bs[k][nn] = (n0 + nn < N && kk + k < K) ? ldc<R>(Bm, (size_t)(n0 + nn) * lda + kk + k) : mk<R>(0, 0);
        }
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < BK; ++k) {
            C a[8], b[4];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = As[k][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[k][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) cfma<R>(acc[i][j], a[i], b[j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        int m = m0 + ty + 16 * i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            int nn = n0 + tx + 16 * j;
            if (nn >= N) continue;
            size_t o = (size_t)nn * lda + m;
            stc<R>(Cm, o, ldc<R>(Cm, o) - acc[i][j]);
        }
    }
}

// ---- triangular solves with the factor of A = Z^T: Z X = B (zgetrs, trans = 'T') -------------------------------------
// U^T y = b (forward, non-unit), L^T z = y (backward, unit), X = P z. B row-major n x nrhs. Blocks of TB rows: the
// block's small triangle solved by one CTA, then the rest of the right-hand sides updated with the block's rows of
// the factor (a contiguous column segment per remaining unknown: coalesced).
#define TB 64
template <typename R>
__global__ void __launch_bounds__(256) k_tri_block(const R *A, long lda, int n, int i0, int bs, R *B, int nrhs, int upper_t)
{
    typedef cpx<R> C;
    extern __shared__ unsigned char tri_raw[];
    C(*T)[TB + 1] = reinterpret_cast<C(*)[TB + 1]>(tri_raw);          // [TB][TB + 1]
    C(*Y)[16] = reinterpret_cast<C(*)[16]>(tri_raw + sizeof(C) * TB * (TB + 1));
    for (int e = threadIdx.x; e < bs * bs; e += blockDim.x) {
        int col = e / bs, row = e % bs;                    // A[i0 + row, i0 + col]
        T[row][col] = ldc<R>(A, (size_t)(i0 + col) * lda + i0 + row);
    }
    for (int e = threadIdx.x; e < bs * nrhs; e += blockDim.x) Y[e / nrhs][e % nrhs] = ldc<R>(B, (size_t)(i0 + e / nrhs) * nrhs + e % nrhs);
    __syncthreads();
    // one thread per right-hand side column (nrhs <= 16)
    if (threadIdx.x < nrhs) {
        int c = threadIdx.x;
        if (upper_t) {          // U^T: lower triangular, T[k][i] = U[k, i] for k < i (column i of U)
            for (int i = 0; i < bs; ++i) {
                C y = Y[i][c];
                for (int k = 0; k < i; ++k) cfms<R>(y, T[k][i], Y[k][c]);
                Y[i][c] = cdiv<R>(y, T[i][i]);
            }
        } else {                // L^T: upper triangular unit, L[k, i] for k > i
            for (int i = bs - 1; i >= 0; --i) {
                C y = Y[i][c];
                for (int k = i + 1; k < bs; ++k) cfms<R>(y, T[k][i], Y[k][c]);
                Y[i][c] = y;
            }
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < bs * nrhs; e += blockDim.x) stc<R>(B, (size_t)(i0 + e / nrhs) * nrhs + e % nrhs, Y[e / nrhs][e % nrhs]);
}

// rest of the right-hand sides: for every unknown i in [lo, hi): B[i] -= sum_{k in block} A[k, i] Y[k]
// (A's column i rows i0..i0+bs: contiguous). One warp per unknown.
template <typename R>
__global__ void __launch_bounds__(256) k_tri_update(const R *A, long lda, int i0, int bs, int lo, int hi, R *B, int nrhs)
{
    typedef cpx<R> C;
    __shared__ C Y[TB][16];
    for (int e = threadIdx.x; e < bs * nrhs; e += blockDim.x) Y[e / nrhs][e % nrhs] = ldc<R>(B, (size_t)(i0 + e / nrhs) * nrhs + e % nrhs);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    for (long i = lo + (blockIdx.x * (long)blockDim.x + threadIdx.x) / 32; i < hi; i += (long)gridDim.x * blockDim.x / 32) {
        C a0 = lane < bs ? ldc<R>(A, (size_t)i * lda + i0 + lane) : mk<R>(0, 0);
        C a1 = lane + 32 < bs ? ldc<R>(A, (size_t)i * lda + i0 + lane + 32) : mk<R>(0, 0);
        for (int c = 0; c < nrhs; ++c) {
            C s = mk<R>(0, 0);
            if (lane < bs) cfma<R>(s, a0, Y[lane][c]);
            if (lane + 32 < bs) cfma<R>(s, a1, Y[lane + 32][c]);
            for (int o = 16; o; o >>= 1) {
                s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
                s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
            }
            if (lane == 0) stc<R>(B, (size_t)i * nrhs + c, ldc<R>(B, (size_t)i * nrhs + c) - s);
        }
    }
}

// X = P z: the interchanges applied from the last to the first (zlaswp with incx = -1): a permutation built in
// shared memory by one thread, then the rows gathered
__global__ void k_perm_from_ipiv(const int *ipiv, int n, int *perm)
{
    extern __shared__ int idx[];
    for (int i = threadIdx.x; i < n; i += blockDim.x) idx[i] = i;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int i = n - 1; i >= 0; --i) {
            int p = ipiv[i];
            if (p < 0 || p >= n) continue;                    // (a failed factorisation: never index past idx)
            int t = idx[i]; idx[i] = idx[p]; idx[p] = t;
        }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = idx[i];
}

template <typename R>
__global__ void k_gather_rows(const R *src, R *dst, const int *perm, int n, int nrhs)
{
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)n * nrhs) return;
    int r = e / nrhs, c = e % nrhs;
    stc<R>(dst, e, ldc<R>(src, (size_t)perm[r] * nrhs + c));
}

// ======================================================================================================================
static int sm_count()
{
    int dev, sms;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    return sms;
}

extern "C" size_t m25_getrf_workspace(int n, int single)
{
    int G = sm_count();
    if (G <= 0) G = 148;
    size_t b = 0;
    b += 2 * (size_t)G * sizeof(double) + 256;                      // cand_val
    b += 2 * (size_t)G * sizeof(int) + 256;                         // cand_idx
    b += 2 * (size_t)G * NB * 2 * sizeof(double) + 256;             // cand_row
    b += 2 * NB * 2 * sizeof(double) + 256;                         // drow
    b += 2 * sizeof(unsigned) + 256;                                // barrier
    if (single) b += m25_umma_workspace(n, NB) + 256;
    (void)n;
    return b;
}

template <typename R>
static int getrf_impl(R *A, long lda, int n, int *ipiv, int tf32, void *work, size_t work_bytes, cudaStream_t s)
{
    int G = sm_count();
    M25_REQUIRE(G > 0, "m25_getrf: no CUDA device");
    M25_REQUIRE(work_bytes >= m25_getrf_workspace(n, sizeof(R) == 4), "m25_getrf: workspace too small");
    int per_sm = 0;
    M25_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_panel<R>, PANEL_THREADS, 0));
    M25_REQUIRE(per_sm >= 1, "m25_getrf: the panel kernel cannot be resident");
    unsigned char *w = (unsigned char *)work;
    auto take = [&](size_t bytes) { unsigned char *p = w; w += (bytes + 255) / 256 * 256; return (void *)p; };
    PanelWork pw;
    pw.cand_val = (double *)take(2 * (size_t)G * sizeof(double));
    pw.cand_idx = (int *)take(2 * (size_t)G * sizeof(int));
    pw.cand_row = (double *)take(2 * (size_t)G * NB * 2 * sizeof(double));
    pw.drow = (double *)take(2 * NB * 2 * sizeof(double));
    unsigned *bar = (unsigned *)take(2 * sizeof(unsigned));
    void *umma_work = take(0);
    size_t umma_bytes = work_bytes - ((unsigned char *)umma_work - (unsigned char *)work);
    pw.bar.count = bar; pw.bar.gen = bar + 1;
    int *err = m25_dev_err_word();
    M25_CHECK(cudaMemsetAsync(ipiv, 0xff, sizeof(int) * (size_t)n, s));      // -1 until the panel sets it
    const size_t trsm_smem = sizeof(cpx<R>) * (NB * NB + NB * 64);
    M25_CHECK(cudaFuncSetAttribute(k_trsm<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem));
    for (int k0 = 0; k0 < n; k0 += NB) {
        const int jb = std::min(NB, n - k0);
        int Gp = std::min(G, std::max(1, (n - k0 + 63) / 64));
        M25_CHECK(cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), s));
        void *args[] = {&A, &lda, &n, (void *)&k0, (void *)&jb, &ipiv, &pw, &err};
        M25_CHECK(cudaLaunchCooperativeKernel((void *)k_panel<R>, dim3(Gp), dim3(PANEL_THREADS), args, 0, s));
        if (n - jb > 0) {
            long cols = n - jb;
            k_laswp<R><<<(cols + 127) / 128, 128, 0, s>>>(A, lda, n, k0, jb, ipiv);
            M25_LAUNCH_CHECK("k_laswp");
        }
        const int rest = n - k0 - jb;
        if (rest > 0) {
            k_trsm<R><<<(rest + 63) / 64, 64, trsm_smem, s>>>(A, lda, n, k0, jb);
            M25_LAUNCH_CHECK("k_trsm");
            R *C22 = A + 2 * ((size_t)(k0 + jb) * lda + k0 + jb);
            const R *L21 = A + 2 * ((size_t)k0 * lda + k0 + jb);
            const R *U12 = A + 2 * ((size_t)(k0 + jb) * lda + k0);
            if (sizeof(R) == 4 && tf32) {
                int rc = m25_umma_trailing((float *)C22, lda, rest, rest, jb, (const float *)L21, (const float *)U12,
                                           umma_work, umma_bytes, s);
                if (rc) return rc;
            } else {
                dim3 grid((rest + 63) / 64, (rest + 127) / 128);
                k_gemm_update<R><<<grid, 256, 0, s>>>(C22, L21, U12, lda, rest, rest, jb);
                M25_LAUNCH_CHECK("k_gemm_update");
            }
        }
    }
    return M25_OK;
}

extern "C" int m25_getrf(void *d_A, long lda, int n, int *d_ipiv, int single, int tf32, void *d_work, size_t work_bytes,
                         void *stream)
{
    M25_REQUIRE(d_A && d_ipiv && d_work && n >= 1 && lda >= n, "m25_getrf: A, ipiv, work, n >= 1, lda >= n");
    M25_REQUIRE(!tf32 || single, "m25_getrf: tf32 updates are for complex64");
    int rc = single ? getrf_impl<float>((float *)d_A, lda, n, d_ipiv, tf32, d_work, work_bytes, S(stream))
                    : getrf_impl<double>((double *)d_A, lda, n, d_ipiv, 0, d_work, work_bytes, S(stream));
    if (rc) return rc;
    return M25_OK;
}

template <typename R>
static int getrs_impl(const R *A, long lda, int n, const int *ipiv, R *B, int nrhs, cudaStream_t s)
{
    const int sms = std::max(1, sm_count());
    const size_t tri_smem = sizeof(cpx<R>) * (TB * (TB + 1) + TB * 16);
    M25_CHECK(cudaFuncSetAttribute(k_tri_block<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tri_smem));
    for (int i0 = 0; i0 < n; i0 += TB) {                              // U^T y = b
        int bs = std::min(TB, n - i0);
        k_tri_block<R><<<1, 256, tri_smem, s>>>(A, lda, n, i0, bs, B, nrhs, 1);
        M25_LAUNCH_CHECK("k_tri_block");
        if (i0 + bs < n) {
            int blocks = std::min(sms * 8, (n - i0 - bs + 7) / 8);
            k_tri_update<R><<<blocks, 256, 0, s>>>(A, lda, i0, bs, i0 + bs, n, B, nrhs);
            M25_LAUNCH_CHECK("k_tri_update");
        }
    }
    for (int i0 = ((n - 1) / TB) * TB; i0 >= 0; i0 -= TB) {           // L^T z = y
        int bs = std::min(TB, n - i0);
        k_tri_block<R><<<1, 256, tri_smem, s>>>(A, lda, n, i0, bs, B, nrhs, 0);
        M25_LAUNCH_CHECK("k_tri_block");
        if (i0 > 0) {
            int blocks = std::min(sms * 8, (i0 + 7) / 8);
            k_tri_update<R><<<blocks, 256, 0, s>>>(A, lda, i0, bs, 0, i0, B, nrhs);
            M25_LAUNCH_CHECK("k_tri_update");
        }
    }
    // X = P z
    int *perm;
    R *tmp;
    M25_CHECK(cudaMallocAsync(&perm, sizeof(int) * n, s));
    M25_CHECK(cudaMallocAsync(&tmp, sizeof(R) * 2 * (size_t)n * nrhs, s));
    M25_REQUIRE(sizeof(int) * (size_t)n <= 200 * 1024, "m25_getrs: n above 51200");
    M25_CHECK(cudaFuncSetAttribute(k_perm_from_ipiv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(sizeof(int) * n)));
    k_perm_from_ipiv<<<1, 1024, sizeof(int) * n, s>>>(ipiv, n, perm);
    M25_LAUNCH_CHECK("k_perm_from_ipiv");
    M25_CHECK(cudaMemcpyAsync(tmp, B, sizeof(R) * 2 * (size_t)n * nrhs, cudaMemcpyDeviceToDevice, s));
    long tot = (long)n * nrhs;
    k_gather_rows<R><<<(tot + 255) / 256, 256, 0, s>>>(tmp, B, perm, n, nrhs);
    M25_LAUNCH_CHECK("k_gather_rows");
    M25_CHECK(cudaFreeAsync(perm, s));
    M25_CHECK(cudaFreeAsync(tmp, s));
    return M25_OK;
}

extern "C" int m25_getrs(const void *d_LU, long lda, int n, const int *d_ipiv, int single, void *d_B, int nrhs, void *stream)
{
    M25_REQUIRE(d_LU && d_ipiv && d_B && n >= 1 && lda >= n, "m25_getrs: LU, ipiv, B, n >= 1");
    M25_REQUIRE(nrhs >= 1 && nrhs <= 16, "m25_getrs: 1 to 16 right-hand sides a call");
    return single ? getrs_impl<float>((const float *)d_LU, lda, n, d_ipiv, (float *)d_B, nrhs, S(stream))
                  : getrs_impl<double>((const double *)d_LU, lda, n, d_ipiv, (double *)d_B, nrhs, S(stream));
}
