// gmres.cu - the vector kernels of the mixed-precision refinement (mom25d fast.py:1437-1500 gmres_batched, run in
// lockstep over k right-hand sides) and the pieces of the exact double-precision operator it iterates with
// (fast.py:571-593 matvec_exact): the near-field COO product and the via border.
// Vectors are N x k row-major complex128 (one column per right-hand side).
#include "common.cuh"

static inline cudaStream_t S(void *s) { return (cudaStream_t)s; }

// out[c] = sum_n conj(V[n, c]) W[n, c]  (out zeroed by the caller; block partial sums added atomically)
__global__ void k_dotc_cols(const double *V, const double *W, long N, int k, double *out)
{
    __shared__ double sx[16][33], sy[16][33];
    double ax[16], ay[16];
    for (int c = 0; c < 16; ++c) ax[c] = ay[c] = 0;
    for (long n = blockIdx.x * (long)blockDim.x + threadIdx.x; n < N; n += (long)gridDim.x * blockDim.x)
        for (int c = 0; c < k; ++c) {
            zd v = ldc<double>(V, (size_t)n * k + c), w = ldc<double>(W, (size_t)n * k + c);
            ax[c] += v.x * w.x + v.y * w.y;
            ay[c] += v.x * w.y - v.y * w.x;
        }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int c = 0; c < k; ++c) {
        double x = ax[c], y = ay[c];
        for (int o = 16; o; o >>= 1) { x += __shfl_xor_sync(0xffffffffu, x, o); y += __shfl_xor_sync(0xffffffffu, y, o); }
        if (lane == 0) { sx[c][wid] = x; sy[c][wid] = y; }
    }
    __syncthreads();
    if (threadIdx.x < k) {
        double x = 0, y = 0;
        for (int j = 0; j < (int)(blockDim.x / 32); ++j) { x += sx[threadIdx.x][j]; y += sy[threadIdx.x][j]; }
        atomicAdd(out + 2 * threadIdx.x, x);
        atomicAdd(out + 2 * threadIdx.x + 1, y);
    }
}

// W[n, c] += V[n, c] a[c]   (a complex, per column)
__global__ void k_axpy_cols(double *W, const double *V, const double *a, long N, int k)
{
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= N * k) return;
    int c = e % k;
    zd w = ldc<double>(W, e);
    cfma<double>(w, ldc<double>(V, e), ldc<double>(a, c));
    stc<double>(W, e, w);
}

// Y[n, c] = X[n, c] s[c] (s complex per column) and, with d != NULL, times d[n] (a row scaling)
__global__ void k_scale_cols(double *Y, const double *X, const double *s, const double *d, long N, int k)
{
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= N * k) return;
    int c = e % k;
    long n = e / k;
    zd x = ldc<double>(X, e);
    if (s) x = x * ldc<double>(s, c);
    if (d) x = x * d[n];
    stc<double>(Y, e, x);
}

// complex128 <-> complex64 (the complex64 factor's solves)
__global__ void k_z2c(const double *X, float *Y, long n)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) { Y[2 * i] = (float)X[2 * i]; Y[2 * i + 1] = (float)X[2 * i + 1]; }
}
__global__ void k_c2z(const float *X, double *Y, long n)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) { Y[2 * i] = X[2 * i]; Y[2 * i + 1] = X[2 * i + 1]; }
}

// Y[ri[s], c] += vv[s] X[ci[s], c] over the near field's COO triplets (ri < 0: unused)
__global__ void k_coo_spmm(const int *ri, const int *ci, const double *vv, long nnz, const double *X, int k, double *Y)
{
    long s = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (s >= nnz) return;
    int r = ri[s];
    if (r < 0) return;
    int cc = ci[s];
    zd v = ldc<double>(vv, s);
    for (int c = 0; c < k; ++c) {
        zd y = v * ldc<double>(X, (size_t)cc * k + c);
        atomicAdd(Y + 2 * ((size_t)r * k + c), y.x);
        atomicAdd(Y + 2 * ((size_t)r * k + c) + 1, y.y);
    }
}

// Y[e, c] += sum over the near field's triplets of row e of vv X[col, c], one warp per edge e. Row e's triplets are
// the slots 9 i + 3 s + u of the pairs i whose observation triangle is one of e's two triangles (the pairs are sorted
// by it: off[t] .. off[t + 1]), s the slot of e on that triangle; the column is te[3 Q[i] + u]. A fixed order:
// deterministic sums, no atomics.
__global__ void k_near_rows_spmm(m25_mesh g, const long long *off, const int *Q, const double *vv, const double *X,
                                 int k, double *Y)
{
    const int e = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
    if (e >= g.Ne) return;
    double ax[16], ay[16];
    for (int c = 0; c < 16; ++c) ax[c] = ay[c] = 0;
    for (int h = 0; h < 2; ++h) {
        const int t = h ? g.em[e] : g.ep[e];
        int s = 0;
        while (s < 3 && g.te[3 * t + s] != e) ++s;
        if (s == 3) continue;
        const long long i0 = off[t], i1 = off[t + 1];
        for (long long j = i0 * 3 + lane; j < i1 * 3; j += 32) {
            const long long i = j / 3;
            const int u = (int)(j % 3);
            const int col = g.te[3 * Q[i] + u];
            if (col < 0) continue;
            const zd v = ldc<double>(vv, (size_t)(9 * i + 3 * s + u));
            for (int c = 0; c < k; ++c) {
                const zd x = ldc<double>(X, (size_t)col * k + c);
                ax[c] = fma(v.x, x.x, ax[c]); ax[c] = fma(-v.y, x.y, ax[c]);
                ay[c] = fma(v.x, x.y, ay[c]); ay[c] = fma(v.y, x.x, ay[c]);
            }
        }
    }
    for (int c = 0; c < k; ++c) {
        double x = ax[c], y = ay[c];
        for (int o = 16; o; o >>= 1) { x += __shfl_xor_sync(0xffffffffu, x, o); y += __shfl_xor_sync(0xffffffffu, y, o); }
        if (lane == 0) {
            zd cur = ldc<double>(Y, (size_t)e * k + c);
            stc<double>(Y, (size_t)e * k + c, cur + mk<double>(x, y));
        }
    }
}

// Z (complex64, ld) += vv at (ri, ci) (the near field into the mixed-precision matrix)
__global__ void k_coo_add_c64(const int *ri, const int *ci, const double *vv, long nnz, float *Z, long ld)
{
    long s = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (s >= nnz) return;
    int r = ri[s];
    if (r < 0) return;
    zd v = ldc<double>(vv, s);
    size_t o = (size_t)r * ld + ci[s];
    atomicAdd(Z + 2 * o, (float)v.x);
    atomicAdd(Z + 2 * o + 1, (float)v.y);
}

// the via border of Z X (fast.py:580-586 _bordered): Y[:Ne] += B X[Ne:], Y[Ne:] = B^T X[:Ne] + C X[Ne:]
// B: Ne x Nv, C: Nv x Nv row-major complex128
__global__ void k_border_top(const double *B, int Ne, int Nv, const double *X, int k, double *Y)
{
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)Ne * k) return;
    long r = e / k;
    int c = e % k;
    zd acc = ldc<double>(Y, e);
    for (int n = 0; n < Nv; ++n) cfma<double>(acc, ldc<double>(B, (size_t)r * Nv + n), ldc<double>(X, (size_t)(Ne + n) * k + c));
    stc<double>(Y, e, acc);
}
__global__ void k_border_bottom(const double *B, const double *C, int Ne, int Nv, const double *X, int k, double *Y)
{
    // one block per (n, c): B^T X over the Ne edges, reduced in the block
    int n = blockIdx.x / k, c = blockIdx.x % k;
    zd acc = mk<double>(0, 0);
    for (long e = threadIdx.x; e < Ne; e += blockDim.x) cfma<double>(acc, ldc<double>(B, (size_t)e * Nv + n), ldc<double>(X, (size_t)e * k + c));
    __shared__ double sx[32], sy[32];
    double x = acc.x, y = acc.y;
    for (int o = 16; o; o >>= 1) { x += __shfl_xor_sync(0xffffffffu, x, o); y += __shfl_xor_sync(0xffffffffu, y, o); }
    if ((threadIdx.x & 31) == 0) { sx[threadIdx.x >> 5] = x; sy[threadIdx.x >> 5] = y; }
    __syncthreads();
    if (threadIdx.x == 0) {
        zd t = mk<double>(0, 0);
        for (int j = 0; j < (int)(blockDim.x / 32); ++j) t += mk<double>(sx[j], sy[j]);
        for (int m = 0; m < Nv; ++m) cfma<double>(t, ldc<double>(C, (size_t)n * Nv + m), ldc<double>(X, (size_t)(Ne + m) * k + c));
        stc<double>(Y, (size_t)(Ne + n) * k + c, t);
    }
}

// Y (n x k) = Z (n x n, row-major, leading dimension ld) X (n x k), complex128, k <= KMAX: the dense double-precision
// product of the refinement when the double Z is resident (fast.py:1009 _solve_kept, A = Z @ V). Streams Z once
// (HBM-bound). A block takes 8 warps x RW rows; X is staged in shared memory a chunk of JC rows at a time, column-
// major (conflict-free reads), and every X value loaded from shared memory serves the warp's RW rows.
__device__ __forceinline__ void cp_async16_zfill(void *smem, const void *gmem, bool valid)
{
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sa), "l"(gmem), "r"(valid ? 16 : 0) : "memory");
}

template <int KMAX>
constexpr int zgemm_jc() { return KMAX >= 16 ? 128 : 256; }

// 16 columns: two rows a warp in the registers of one CTA an SM (4.14 ms at N = 18,788 against 5.32 for one row at
// two CTAs an SM, which spilled); up to 8 columns two CTAs an SM (8 columns with four rows at one CTA: 674 against
// 619 us at N = 9,600)
template <int KMAX, int RW>
__global__ void __launch_bounds__(256, RW * KMAX >= 32 ? 1 : 2) k_zgemm_skinny(const double *__restrict__ Z, long ld, int n,
                                                         const double *__restrict__ X, int k, double *__restrict__ Y)
{
    constexpr int JC = zgemm_jc<KMAX>();
    extern __shared__ __align__(16) double2 xs_dyn[];                  // [2][KMAX * JC], column-major chunks
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long row0 = ((long)blockIdx.x * 8 + warp) * RW;
    double2 acc[RW][KMAX];
#pragma unroll
    for (int r = 0; r < RW; ++r)
#pragma unroll
        for (int c = 0; c < KMAX; ++c) acc[r][c] = make_double2(0.0, 0.0);
    const double2 *Z2 = reinterpret_cast<const double2 *>(Z);
    const double2 *X2 = reinterpret_cast<const double2 *>(X);
    // X chunk j0 .. j0 + JC into buffer buf by cp.async (zero past n and past k columns)
    auto stage = [&](int buf, int j0) {
        double2 *dst = xs_dyn + (size_t)buf * KMAX * JC;
        for (int e = threadIdx.x; e < JC * KMAX; e += 256) {
            const int j = e / KMAX, c = e % KMAX;
            const bool ok = c < k && j0 + j < n;
            cp_async16_zfill(dst + c * JC + j, X2 + (ok ? (size_t)(j0 + j) * k + c : 0), ok);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    stage(0, 0);
    int it = 0;
    for (int j0 = 0; j0 < n; j0 += JC, ++it) {
        const int jn = min(JC, n - j0);
        if (j0 + JC < n) stage((it + 1) & 1, j0 + JC);                   // the next chunk, other buffer
        else asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 1;" ::: "memory");            // this chunk has landed
        __syncthreads();
        const double2 *xs = xs_dyn + (size_t)(it & 1) * KMAX * JC;
#pragma unroll 4
        for (int q = 0; q < JC / 32; ++q) {
            const int jj = q * 32 + lane;
            double2 z[RW];
#pragma unroll
            for (int r = 0; r < RW; ++r)
                z[r] = (jj < jn && row0 + r < n) ? __ldcs(Z2 + (size_t)(row0 + r) * ld + j0 + jj) : make_double2(0.0, 0.0);
#pragma unroll
            for (int c = 0; c < KMAX; ++c) {                                // (columns past k are zero in xs)
                const double2 x = xs[c * JC + jj];
#pragma unroll
                for (int r = 0; r < RW; ++r) {
                    acc[r][c].x = fma(z[r].x, x.x, fma(-z[r].y, x.y, acc[r][c].x));
                    acc[r][c].y = fma(z[r].x, x.y, fma(z[r].y, x.x, acc[r][c].y));
                }
            }
        }
        __syncthreads();                                                 // the buffer is the chunk after next's
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
#pragma unroll
    for (int r = 0; r < RW; ++r)
#pragma unroll
        for (int c = 0; c < KMAX; ++c) {
            double a = acc[r][c].x, b = acc[r][c].y;
#pragma unroll
            for (int o = 16; o; o >>= 1) { a += __shfl_xor_sync(0xffffffffu, a, o); b += __shfl_xor_sync(0xffffffffu, b, o); }
            if (lane == c && c < k && row0 + r < n) reinterpret_cast<double2 *>(Y)[(size_t)(row0 + r) * k + c] = make_double2(a, b);
        }
}

template <int KMAX, int RW>
static int zgemm_launch(const double *d_Z, long ld, int n, const double *d_X, int k, double *d_Y, cudaStream_t s)
{
    const int smem = (int)(2 * sizeof(double2) * KMAX * zgemm_jc<KMAX>());
    if (smem > 48 * 1024) M25_CHECK(cudaFuncSetAttribute(k_zgemm_skinny<KMAX, RW>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_zgemm_skinny<KMAX, RW><<<(unsigned)((n + 8 * RW - 1) / (8 * RW)), 256, smem, s>>>(d_Z, ld, n, d_X, k, d_Y);
    M25_LAUNCH_CHECK("k_zgemm_skinny");
    return M25_OK;
}

// The same product for up to 8 columns on the FP64 tensor cores (above 4 columns the CUDA-core kernel is bound by
// its four FP64 FMAs a complex term, not by HBM): a warp takes 16 rows of Z and walks its share of the row in steps
// of 8 columns, one m16n8k8 f64 MMA per real part (Yr += Zr Xr - Zi Xi, Yi += Zr Xi + Zi Xr). The MMA's K slots are
// matched to the columns as slot t <-> column 2 t, slot t + 4 <-> column 2 t + 1 (the same in A and in B), so that
// each lane reads two adjacent complex entries (32 bytes) of its two rows and the four lanes of a row 128 contiguous
// bytes; UNR steps of loads are issued before their MMAs. X (read by every warp) comes through the read-only cache.
// ks warps (1, 2 or 4) share a group of 16 rows, each a contiguous share of the columns, their partial sums added
// through shared memory, so that small n still fills the SMs. kk <= 8 columns of X and Y, row strides ldx and ldy
// (a 16-column product is two such passes).
template <int UNR>
__global__ void __launch_bounds__(256, 1) k_zgemm_dmma8(const double *__restrict__ Z, long ld, int n,
                                                        const double *__restrict__ X, int kk, int ldx,
                                                        double *__restrict__ Y, int ldy, int ks)
{
    __shared__ double red[8][32][8];                                  // [warp][lane][dr 0..3, di 0..3]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    const int rg = warp / ks, part = warp % ks;
    const long row0 = ((long)blockIdx.x * (8 / ks) + rg) * 16;
    const double2 *Z2 = reinterpret_cast<const double2 *>(Z);
    const double2 *X2 = reinterpret_cast<const double2 *>(X);
    const long ra = row0 + g, rb = row0 + g + 8;
    const bool va = ra < n, vb = rb < n, colok = g < kk;
    const double2 *za = Z2 + (size_t)(va ? ra : 0) * ld, *zb = Z2 + (size_t)(vb ? rb : 0) * ld;
    const double2 zero = make_double2(0.0, 0.0);
    double dr[4] = {0, 0, 0, 0}, di[4] = {0, 0, 0, 0};
    const long step = 8L * UNR, share = ((n + step - 1) / step + ks - 1) / ks * step;
    const long jbeg = part * share, jend = min((long)n, jbeg + share);
    for (long j0 = row0 < n ? jbeg : jend; j0 < jend; j0 += step) {
        double2 a[UNR][4], b[UNR][2];
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const long j = j0 + 8 * u + 2 * t;
            const bool j0ok = j < jend, j1ok = j + 1 < jend;
            a[u][0] = va && j0ok ? __ldcs(za + j) : zero;                 // A[g][t]
            a[u][1] = vb && j0ok ? __ldcs(zb + j) : zero;                 // A[g + 8][t]
            a[u][2] = va && j1ok ? __ldcs(za + j + 1) : zero;             // A[g][t + 4]
            a[u][3] = vb && j1ok ? __ldcs(zb + j + 1) : zero;             // A[g + 8][t + 4]
            b[u][0] = colok && j0ok ? __ldg(X2 + (size_t)j * ldx + g) : zero;        // B[t][g]
            b[u][1] = colok && j1ok ? __ldg(X2 + (size_t)(j + 1) * ldx + g) : zero;  // B[t + 4][g]
        }
#pragma unroll
        for (int u = 0; u < UNR; ++u) {
            const double ar[4] = {a[u][0].x, a[u][1].x, a[u][2].x, a[u][3].x};
            const double ai[4] = {a[u][0].y, a[u][1].y, a[u][2].y, a[u][3].y};
            const double br[2] = {b[u][0].x, b[u][1].x}, bi[2] = {b[u][0].y, b[u][1].y};
            const double nbi[2] = {-b[u][0].y, -b[u][1].y};
            dmma_16x8x8(dr, ar, br);
            dmma_16x8x8(dr, ai, nbi);
            dmma_16x8x8(di, ar, bi);
            dmma_16x8x8(di, ai, br);
        }
    }
    if (ks > 1) {                                                     // the row group's shares added by its first warp
#pragma unroll
        for (int q = 0; q < 4; ++q) { red[warp][lane][q] = dr[q]; red[warp][lane][4 + q] = di[q]; }
        __syncthreads();
        if (part != 0) return;
        for (int p = 1; p < ks; ++p)
#pragma unroll
            for (int q = 0; q < 4; ++q) { dr[q] += red[warp + p][lane][q]; di[q] += red[warp + p][lane][4 + q]; }
    }
    double2 *Y2 = reinterpret_cast<double2 *>(Y);                    // D[g][2t], D[g][2t + 1], D[g + 8][2t], ...
    const int c0 = 2 * t, c1 = 2 * t + 1;
    if (va && c0 < kk) Y2[(size_t)ra * ldy + c0] = make_double2(dr[0], di[0]);
    if (va && c1 < kk) Y2[(size_t)ra * ldy + c1] = make_double2(dr[1], di[1]);
    if (vb && c0 < kk) Y2[(size_t)rb * ldy + c0] = make_double2(dr[2], di[2]);
    if (vb && c1 < kk) Y2[(size_t)rb * ldy + c1] = make_double2(dr[3], di[3]);
}

// ks: the fewest warps a row group that give three quarters of the SMs or more a CTA (8 warps an SM)
static int zdmma8_launch(const double *d_Z, long ld, int n, const double *d_X, int kk, int ldx, double *d_Y, int ldy,
                         cudaStream_t s)
{
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        M25_CHECK(cudaGetDevice(&dev));
        M25_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    }
    const long groups = (n + 15) / 16;
    int ks = 1;
    while (ks < 4 && 4 * ((groups * ks + 7) / 8) < 3 * (long)sms) ks *= 2;
    const long ctas = (groups * ks + 7) / 8;
    k_zgemm_dmma8<4><<<(unsigned)ctas, 256, 0, s>>>(d_Z, ld, n, d_X, kk, ldx, d_Y, ldy, ks);
    M25_LAUNCH_CHECK("k_zgemm_dmma8");
    return M25_OK;
}

// The Gram-Schmidt step of the batched GMRES against all basis vectors at once (classical Gram-Schmidt, applied
// twice by the caller): out[i, c] = sum_n conj(V_i[n, c]) W[n, c] for i < nv (V: nv consecutive N x k blocks), one
// grid row of blocks per vector; W -= sum_i V_i h[i] (h: nv x k complex, per column).
__global__ void k_dotc_multi(const double *V, long N, int k, const double *W, double *out)
{
    const double *Vi = V + 2 * (size_t)blockIdx.y * N * k;
    __shared__ double sx[16][33], sy[16][33];
    double ax[16], ay[16];
    for (int c = 0; c < 16; ++c) ax[c] = ay[c] = 0;
    for (long n = blockIdx.x * (long)blockDim.x + threadIdx.x; n < N; n += (long)gridDim.x * blockDim.x)
        for (int c = 0; c < k; ++c) {
            zd v = ldc<double>(Vi, (size_t)n * k + c), w = ldc<double>(W, (size_t)n * k + c);
            ax[c] += v.x * w.x + v.y * w.y;
            ay[c] += v.x * w.y - v.y * w.x;
        }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int c = 0; c < k; ++c) {
        double x = ax[c], y = ay[c];
        for (int o = 16; o; o >>= 1) { x += __shfl_xor_sync(0xffffffffu, x, o); y += __shfl_xor_sync(0xffffffffu, y, o); }
        if (lane == 0) { sx[c][wid] = x; sy[c][wid] = y; }
    }
    __syncthreads();
    if (threadIdx.x < k) {
        double x = 0, y = 0;
        for (int j = 0; j < (int)(blockDim.x / 32); ++j) { x += sx[threadIdx.x][j]; y += sy[threadIdx.x][j]; }
        atomicAdd(out + 2 * ((size_t)blockIdx.y * k + threadIdx.x), x);
        atomicAdd(out + 2 * ((size_t)blockIdx.y * k + threadIdx.x) + 1, y);
    }
}

__global__ void k_axpy_multi(double *W, const double *V, int nv, long N, int k, const double *h)
{
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= N * k) return;
    const int c = e % k;
    zd w = ldc<double>(W, e);
    for (int i = 0; i < nv; ++i) cfms<double>(w, ldc<double>(V, (size_t)i * N * k + e), ldc<double>(h, (size_t)i * k + c));
    stc<double>(W, e, w);
}

// ======================================================================================================================
extern "C" int m25_dotc_cols(const double *d_V, const double *d_W, long N, int k, double *d_out, void *stream)
{
    M25_REQUIRE(k >= 1 && k <= 16, "m25_dotc_cols: 1 to 16 columns");
    M25_CHECK(cudaMemsetAsync(d_out, 0, sizeof(double) * 2 * k, S(stream)));
    int blocks = (int)std::min<long>(592, (N + 255) / 256);
    k_dotc_cols<<<blocks, 256, 0, S(stream)>>>(d_V, d_W, N, k, d_out);
    M25_LAUNCH_CHECK("k_dotc_cols");
    return M25_OK;
}

extern "C" int m25_axpy_cols(double *d_W, const double *d_V, const double *d_a, long N, int k, void *stream)
{
    long t = N * k;
    k_axpy_cols<<<(t + 255) / 256, 256, 0, S(stream)>>>(d_W, d_V, d_a, N, k);
    M25_LAUNCH_CHECK("k_axpy_cols");
    return M25_OK;
}

extern "C" int m25_scale_cols(double *d_Y, const double *d_X, const double *d_s, const double *d_rows, long N, int k,
                              void *stream)
{
    long t = N * k;
    k_scale_cols<<<(t + 255) / 256, 256, 0, S(stream)>>>(d_Y, d_X, d_s, d_rows, N, k);
    M25_LAUNCH_CHECK("k_scale_cols");
    return M25_OK;
}

extern "C" int m25_convert(const void *d_in, int in_single, void *d_out, long n, void *stream)
{
    if (!n) return M25_OK;
    if (in_single) k_c2z<<<(n + 255) / 256, 256, 0, S(stream)>>>((const float *)d_in, (double *)d_out, n);
    else k_z2c<<<(n + 255) / 256, 256, 0, S(stream)>>>((const double *)d_in, (float *)d_out, n);
    M25_LAUNCH_CHECK("k_convert");
    return M25_OK;
}

extern "C" int m25_coo_spmm(const int *d_ri, const int *d_ci, const double *d_vv, long nnz, const double *d_X, int k,
                            double *d_Y, void *stream)
{
    if (!nnz) return M25_OK;
    k_coo_spmm<<<(nnz + 255) / 256, 256, 0, S(stream)>>>(d_ri, d_ci, d_vv, nnz, d_X, k, d_Y);
    M25_LAUNCH_CHECK("k_coo_spmm");
    return M25_OK;
}

extern "C" int m25_near_spmm_rows(const m25_mesh *g, const long long *d_off, const int *d_Q, const double *d_vv,
                                  const double *d_X, int k, double *d_Y, void *stream)
{
    M25_REQUIRE(g && k >= 1 && k <= 16, "m25_near_spmm_rows: mesh, 1 to 16 columns");
    if (!g->Ne) return M25_OK;
    k_near_rows_spmm<<<(g->Ne + 7) / 8, 256, 0, S(stream)>>>(*g, d_off, d_Q, d_vv, d_X, k, d_Y);
    M25_LAUNCH_CHECK("k_near_rows_spmm");
    return M25_OK;
}

extern "C" int m25_coo_add_c64(const int *d_ri, const int *d_ci, const double *d_vv, long nnz, float *d_Z, long ld,
                               void *stream)
{
    if (!nnz) return M25_OK;
    k_coo_add_c64<<<(nnz + 255) / 256, 256, 0, S(stream)>>>(d_ri, d_ci, d_vv, nnz, d_Z, ld);
    M25_LAUNCH_CHECK("k_coo_add_c64");
    return M25_OK;
}

int *m25_dev_err_word();

// Z (row-major, ld) += vv at (ri, ci), every (ri, ci) distinct (no atomics: one thread an entry), complex128 or
// complex64 (rounded on store)
template <typename R>
__global__ void k_coo_add_unique(const int *ri, const int *ci, const double *vv, long nnz, R *Z, long ld, long n,
                                 int *err)
{
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= nnz) return;
    const long r = ri[e], c = ci[e];
    if (r < 0 || r >= n || c < 0 || c >= n) { dev_error(err, M25_DEV_INDEX); return; }
    const size_t o = 2 * ((size_t)r * ld + c);
    Z[o] = (R)((double)Z[o] + vv[2 * e]);
    Z[o + 1] = (R)((double)Z[o + 1] + vv[2 * e + 1]);
}

extern "C" int m25_coo_add(const int *d_ri, const int *d_ci, const double *d_vv, long nnz, void *d_Z, long ld,
                           int n, int single, void *stream)
{
    M25_REQUIRE(nnz >= 0 && (!nnz || (d_ri && d_ci && d_vv && d_Z)) && n >= 0 && ld >= n,
                "m25_coo_add: ri, ci, vv, Z, nnz >= 0, ld >= n");
    if (!nnz) return M25_OK;
    int *err = m25_dev_err_word();
    if (single)
        k_coo_add_unique<float><<<(nnz + 255) / 256, 256, 0, S(stream)>>>(d_ri, d_ci, d_vv, nnz, (float *)d_Z, ld,
                                                                            n, err);
    else
        k_coo_add_unique<double><<<(nnz + 255) / 256, 256, 0, S(stream)>>>(d_ri, d_ci, d_vv, nnz, (double *)d_Z,
                                                                             ld, n, err);
    M25_LAUNCH_CHECK("k_coo_add_unique");
    return M25_OK;
}

extern "C" int m25_border_mv(const double *d_B, const double *d_C, int Ne, int Nv, const double *d_X, int k,
                             double *d_Y, void *stream)
{
    if (!Nv) return M25_OK;
    long t = (long)Ne * k;
    k_border_top<<<(t + 255) / 256, 256, 0, S(stream)>>>(d_B, Ne, Nv, d_X, k, d_Y);
    M25_LAUNCH_CHECK("k_border_top");
    k_border_bottom<<<Nv * k, 256, 0, S(stream)>>>(d_B, d_C, Ne, Nv, d_X, k, d_Y);
    M25_LAUNCH_CHECK("k_border_bottom");
    return M25_OK;
}

extern "C" int m25_zgemm_skinny(const double *d_Z, long ld, int n, const double *d_X, int k, double *d_Y, void *stream)
{
    M25_REQUIRE(d_Z && d_X && d_Y && n >= 0 && ld >= n, "m25_zgemm_skinny: Z, X, Y, ld >= n");
    M25_REQUIRE(k >= 1 && k <= 16, "m25_zgemm_skinny: 1 to 16 columns");
    if (!n) return M25_OK;
    // fewer rows a warp as the columns grow (registers: two CTAs an SM keep enough loads of Z in flight)
    if (k <= 2) return zgemm_launch<2, 4>(d_Z, ld, n, d_X, k, d_Y, S(stream));
    if (k <= 4) return zgemm_launch<4, 4>(d_Z, ld, n, d_X, k, d_Y, S(stream));
    if (const char *e = getenv("M25_ZGEMM_DMMA")) {
        if (atoi(e) == 0) {                                  // (the CUDA-core kernel: comparisons)
            if (k <= 8) return zgemm_launch<8, 2>(d_Z, ld, n, d_X, k, d_Y, S(stream));
            return zgemm_launch<16, 2>(d_Z, ld, n, d_X, k, d_Y, S(stream));
        }
    }
    int rc = zdmma8_launch(d_Z, ld, n, d_X, std::min(k, 8), k, d_Y, k, S(stream));   // columns 0 .. 8
    if (rc || k <= 8) return rc;
    return zdmma8_launch(d_Z, ld, n, d_X + 16, k - 8, k, d_Y + 16, k, S(stream));   // columns 8 .. k
}

extern "C" int m25_dotc_multi(const double *d_V, int nv, long N, int k, const double *d_W, double *d_out, void *stream)
{
    M25_REQUIRE(k >= 1 && k <= 16 && nv >= 1 && nv <= 65535, "m25_dotc_multi: 1 to 16 columns, nv >= 1");
    M25_CHECK(cudaMemsetAsync(d_out, 0, sizeof(double) * 2 * (size_t)nv * k, S(stream)));
    dim3 grid((unsigned)std::min<long>(148, (N + 255) / 256), (unsigned)nv);
    k_dotc_multi<<<grid, 256, 0, S(stream)>>>(d_V, N, k, d_W, d_out);
    M25_LAUNCH_CHECK("k_dotc_multi");
    return M25_OK;
}

extern "C" int m25_axpy_multi(double *d_W, const double *d_V, int nv, long N, int k, const double *d_h, void *stream)
{
    long t = N * k;
    if (!t || nv <= 0) return M25_OK;
    k_axpy_multi<<<(t + 255) / 256, 256, 0, S(stream)>>>(d_W, d_V, nv, N, k, d_h);
    M25_LAUNCH_CHECK("k_axpy_multi");
    return M25_OK;
}

// ---- one Arnoldi step of the batched GMRES on the device ------------------------------------------------------------
// h[i, c] += d[i, c] (n complex coefficients): the second Gram-Schmidt pass's correction
__global__ void k_add_coef(double *h, const double *d, int n)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    h[2 * e] += d[2 * e];
    h[2 * e + 1] += d[2 * e + 1];
}

// V[n, c] = W[n, c] / sqrt(re nrm2[c]) (a zero norm: V = 0, the column has broken down and stays converged)
__global__ void k_scale_rnorm(double *V, const double *W, const double *nrm2, long N, int k)
{
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= N * k) return;
    const double s = nrm2[2 * (e % k)];
    const double r = s > 0 ? rsqrt(s) : 0.0;
    zd w = ldc<double>(W, e);
    stc<double>(V, e, w * r);
}

// nrm2[c] = (sqrt(re nrm2[c]), 0): the subdiagonal entry of the Hessenberg column
__global__ void k_sqrt_norms(double *nrm2, int k)
{
    const int c = threadIdx.x;
    if (c >= k) return;
    nrm2[2 * c] = sqrt(fmax(nrm2[2 * c], 0.0));
    nrm2[2 * c + 1] = 0.0;
}

// W (the operator applied to the j-th preconditioned direction) orthogonalised against the basis blocks
// V_0 .. V_j by classical Gram-Schmidt applied twice, and normalised into V_{j+1}; the Hessenberg column goes to
// h ((j + 2) x k complex: the j + 1 projections, then the norm). tmp: (j + 1) x k complex of scratch. Nothing
// is read back: the host takes h once per step.
extern "C" int m25_arnoldi_orth(double *d_V, int j, long N, int k, double *d_W, double *d_h, double *d_tmp,
                                void *stream)
{
    M25_REQUIRE(d_V && d_W && d_h && d_tmp && j >= 0 && j < 65535 && k >= 1 && k <= 16 && N >= 1,
                "m25_arnoldi_orth: V, W, h, tmp, 0 <= j, 1 to 16 columns");
    cudaStream_t s = S(stream);
    const int nv = j + 1;
    const size_t hb = sizeof(double) * 2 * (size_t)nv * k;
    dim3 grid((unsigned)std::min<long>(148, (N + 255) / 256), (unsigned)nv);
    const long t = N * k;
    M25_CHECK(cudaMemsetAsync(d_h, 0, hb + sizeof(double) * 2 * k, s));
    k_dotc_multi<<<grid, 256, 0, s>>>(d_V, N, k, d_W, d_h);
    M25_LAUNCH_CHECK("k_dotc_multi");
    k_axpy_multi<<<(t + 255) / 256, 256, 0, s>>>(d_W, d_V, nv, N, k, d_h);
    M25_LAUNCH_CHECK("k_axpy_multi");
    M25_CHECK(cudaMemsetAsync(d_tmp, 0, hb, s));
    k_dotc_multi<<<grid, 256, 0, s>>>(d_V, N, k, d_W, d_tmp);
    M25_LAUNCH_CHECK("k_dotc_multi");
    k_axpy_multi<<<(t + 255) / 256, 256, 0, s>>>(d_W, d_V, nv, N, k, d_tmp);
    M25_LAUNCH_CHECK("k_axpy_multi");
    k_add_coef<<<(nv * k + 255) / 256, 256, 0, s>>>(d_h, d_tmp, nv * k);
    M25_LAUNCH_CHECK("k_add_coef");
    double *nrm = d_h + 2 * (size_t)nv * k;
    k_dotc_cols<<<(int)std::min<long>(592, (N + 255) / 256), 256, 0, s>>>(d_W, d_W, N, k, nrm);
    M25_LAUNCH_CHECK("k_dotc_cols");
    k_scale_rnorm<<<(t + 255) / 256, 256, 0, s>>>(d_V + 2 * (size_t)nv * N * k, d_W, nrm, N, k);
    M25_LAUNCH_CHECK("k_scale_rnorm");
    k_sqrt_norms<<<1, 32, 0, s>>>(nrm, k);
    M25_LAUNCH_CHECK("k_sqrt_norms");
    return M25_OK;
}
