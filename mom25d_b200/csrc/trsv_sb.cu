// trsv_sb.cu - the triangular solves of a factor by 256-row diagonal blocks, the chain between blocks cut to one
// product a block (the solves of m25_getrs_aux where they are enabled, m25_sb_enabled).
//
// With A = Z^T = P L U, Z X = B is U^T y = B (forward, lower triangular T = U^T, T[r][k] = A[r * lda + k] for
// k <= r), L^T z = y (backward, upper triangular T = L^T with unit diagonal, T[r][k] = A[r * lda + k] for k > r),
// X = P z. Rows are grouped into blocks q of SB = 256 rows, taken in solve order (forward q = 0, 1, ...; backward
// q = ns - 1, ...); position p of a block is its place in that order, and y_p its solution. With, per block,
//   D_p  = inv(T_pp)                       (the block's diagonal part inverted once per factor),
//   K1_p = D_p T_{p, p-1},  K2_p = D_p T_{p, p-2}   (its coupling with the two blocks solved just before it),
// the substitution y_p = D_p (b_p - sum_{j < p} T_pj y_j) becomes
//   w_p = D_p (b_p - sum_{j <= p-3} T_pj y_j),   u_p = w_p - K2_p y_{p-2},   y_p = u_p - K1_p y_{p-1}:
// once y_{p-1} is known, y_p is one product of a 256 x 256 matrix with the right-hand sides, which the 8 CTAs
// holding the block's 32-row chunks share. Everything else (the updates t -= T y of later blocks, w, u) is done a
// step or more ahead, off the chain.
//
// Setup per factor (m25_sb_prepare): k_sb_dinv forms D_p (by 64-row blocks, from the inverses of the factor's
// 64-row diagonal blocks that k_block_inverses made), k_sb_couple K1_p and K2_p. Solve (m25_sb_solve): one
// persistent cooperative kernel a triangle, k_trsv_sb, its CTAs in two roles so that the chain never waits behind
// the bulk of the updates:
//   - 24 chain CTAs: CTA g takes chunk g % 8 (32 rows) of every third block (blocks g / 8, g / 8 + 3, ...). At
//     step s (once y_s is published) the group of the block at position s + 1 forms its y (then publishes it:
//     values, fence, flag = this call's epoch), the group at s + 2 its u, the group at s + 3 its w (from the t of
//     the block's 8 chunks, waiting for their flags): one product a CTA a step. Before step 0 they form w of the
//     blocks at positions 0-2 from b, and publish y_0.
//   - the other CTAs hold the running right-hand sides t of the chunks (chunk c in CTA 24 + c mod (G - 24)): at
//     step s, t -= T y_s for their chunk of the block at s + 3, then they publish that t, then the same update for
//     their chunks of blocks at s + 4 and later.
// Every matrix tile (32 rows x 64 columns of K1, K2, D or the factor) comes through a ring of shared-memory buffers
// by cp.async, several tiles ahead of the product that reads it, so the chain's product finds its matrix in shared
// memory. Waits only point to work of earlier steps, or of this step before any wait: no cycle; every wait is
// bounded and reports M25_DEV_TIMEOUT.
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "common.cuh"

#define SB 256                 // rows of a diagonal block
#define SBC 32                 // rows of a chunk
#define SB_CPB (SB / SBC)      // chunks a block
#define SB_TB 64               // rows of the factor's diagonal-block inverses (k_block_inverses)
#define SB_KT 64               // columns of a staged tile
#define SB_KTS (SB / SB_KT)    // tiles a task
#define SB_TS 72               // tile row stride (complex): 576 bytes; complex64 rows 16 words apart on the banks
#define SB_NT 512              // threads of the solve kernel
#define SB_TPR (SB_NT / SBC)   // threads a chunk row (16)
#define SB_CHMAX 12            // chunks a CTA at most
#define SB_NR 8                // right-hand sides a solve
#define SB_MIN_N 2048          // smallest n solved this way (below it the chain of 64-row blocks is short)
#define SB_GA 24               // CTAs on the chain's products: 8 chunks x 3 blocks in flight (y, u, w)
static_assert(SBC * SB_NR <= SB_NT, "a chunk's entries one a thread");
static_assert(SB_TPR == 16 && SB_KT % SB_TPR == 0, "16 threads a chunk row, whole terms a tile");

template <typename R> constexpr int sb_xs() { return 36 * 4 / (int)sizeof(cpx<R>); }    // staged vector row stride
// shared memory of the solve kernel with a ring of nbuf tiles
template <typename R> constexpr size_t sb_smem(int nbuf)
{
    return sizeof(cpx<R>) * ((size_t)nbuf * SBC * SB_TS + (size_t)SB * sb_xs<R>() + (size_t)SB_CHMAX * SBC * SB_NR);
}

__device__ __forceinline__ void sb_cp16(void *smem, const void *gmem)
{
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void sb_cp8(void *smem, const void *gmem)
{
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void sb_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void sb_wait_group() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// ---- setup ----------------------------------------------------------------------------------------------------------
// The three matrices of block q, triangle tri (0 forward, 1 backward): mats + ((tri * 3 + m) * ns + q) * SB * SB,
// m = 0 D, 1 K1, 2 K2; each SB x SB row-major. Rows and columns past n: D has ones on their diagonal, zeros
// elsewhere; K1, K2 zeros.
template <typename R>
__host__ __device__ __forceinline__ cpx<R> *sb_mat(cpx<R> *mats, int ns, int tri, int m, int q)
{
    return mats + (((size_t)tri * 3 + m) * ns + q) * SB * SB;
}

// 64 x 64 tile product in shared memory: acc += Xa Xb (Xa, Xb [64][65]); thread t: rows t / 16 + 16 i,
// columns t % 16 + 16 j
template <typename R>
__device__ __forceinline__ void sb_mm64(const cpx<R> *Xa, const cpx<R> *Xb, cpx<R> (&acc)[4][4])
{
    const int tr = threadIdx.x >> 4, tc = threadIdx.x & 15;
#pragma unroll 4
    for (int kk = 0; kk < SB_TB; ++kk) {
        cpx<R> av[4], bv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) av[i] = Xa[(tr + 16 * i) * (SB_TB + 1) + kk];
#pragma unroll
        for (int j = 0; j < 4; ++j) bv[j] = Xb[kk * (SB_TB + 1) + tc + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) cfma<R>(acc[i][j], av[i], bv[j]);
    }
}

// T[r0 + r][c0 + c] (r, c < 64) into dst [64][65]: zero past n
template <typename R>
__device__ __forceinline__ void sb_stage_T(cpx<R> *dst, const cpx<R> *A, long lda, int n, int r0, int c0)
{
    for (int e = threadIdx.x; e < SB_TB * SB_TB; e += blockDim.x) {
        const int r = e / SB_TB, c = e % SB_TB;
        dst[r * (SB_TB + 1) + c] = (r0 + r < n && c0 + c < n) ? A[(size_t)(r0 + r) * lda + c0 + c] : mk<R>(0, 0);
    }
}
// a 64 x 64 block of a row-major SB x SB matrix into dst [64][65]
template <typename R>
__device__ __forceinline__ void sb_stage_M(cpx<R> *dst, const cpx<R> *M, int bi, int bj)
{
    for (int e = threadIdx.x; e < SB_TB * SB_TB; e += blockDim.x) {
        const int r = e / SB_TB, c = e % SB_TB;
        dst[r * (SB_TB + 1) + c] = M[(size_t)(bi * SB_TB + r) * SB + bj * SB_TB + c];
    }
}
// the inverse of the factor's diagonal block b transposed: inv(T_bb) = inv(U_bb)^T (forward) or inv(L_bb)^T
template <typename R>
__device__ __forceinline__ void sb_stage_inv(cpx<R> *dst, const cpx<R> *inv64, int b, int tri)
{
    const cpx<R> *src = inv64 + (size_t)b * 2 * SB_TB * SB_TB + (tri == 0 ? (size_t)SB_TB * SB_TB : 0);
    for (int e = threadIdx.x; e < SB_TB * SB_TB; e += blockDim.x) {
        const int r = e / SB_TB, c = e % SB_TB;
        dst[r * (SB_TB + 1) + c] = src[(size_t)c * SB_TB + r];
    }
}
template <typename R>
__device__ __forceinline__ void sb_store_acc(cpx<R> *M, int bi, int bj, const cpx<R> (&acc)[4][4], R sign)
{
    const int tr = threadIdx.x >> 4, tc = threadIdx.x & 15;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
            M[(size_t)(bi * SB_TB + tr + 16 * i) * SB + bj * SB_TB + tc + 16 * j] = acc[i][j] * sign;
}

// D_q = inv(T_qq) by its 64-row blocks: X_jj = inv(T_jj); forward (lower) X_ij = -X_ii sum_{j <= k < i} T_ik X_kj
// for i = j + 1 .. 3; backward (upper) X_ij = -X_ii sum_{i < k <= j} T_ik X_kj for i = j - 1 .. 0. Grid (4 column
// blocks j, ns, 2 triangles); the CTA's earlier X_kj are read back from the output (its own writes, ordered by
// the block barriers).
template <typename R>
__global__ void __launch_bounds__(256) k_sb_dinv(const cpx<R> *A, long lda, int n, int ns, const cpx<R> *inv64,
                                                 cpx<R> *mats)
{
    typedef cpx<R> C;
    extern __shared__ __align__(16) unsigned char sbd_raw[];
    C *Xa = reinterpret_cast<C *>(sbd_raw), *Xb = Xa + SB_TB * (SB_TB + 1);
    const int j = blockIdx.x, q = blockIdx.y, tri = blockIdx.z;
    const int nb64 = (n + SB_TB - 1) / SB_TB, R0 = q * SB;
    C *D = sb_mat(mats, ns, tri, 0, q);
    auto valid = [&](int i) { return 4 * q + i < nb64; };
    // zero this column block, then the diagonal block
    for (int e = threadIdx.x; e < SB * SB_TB; e += blockDim.x) {
        const int r = e / SB_TB, c = e % SB_TB;
        D[(size_t)r * SB + j * SB_TB + c] = mk<R>(0, 0);
    }
    __syncthreads();
    if (!valid(j)) return;
    sb_stage_inv(Xa, inv64, 4 * q + j, tri);
    __syncthreads();
    for (int e = threadIdx.x; e < SB_TB * SB_TB; e += blockDim.x) {
        const int r = e / SB_TB, c = e % SB_TB;
        D[(size_t)(j * SB_TB + r) * SB + j * SB_TB + c] = Xa[r * (SB_TB + 1) + c];
    }
    __syncthreads();
    const int step = tri == 0 ? 1 : -1;
    for (int i = j + step; i >= 0 && i < 4; i += step) {
        if (!valid(i)) break;                        // (forward: the blocks past n; backward never: i < j)
        C acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = mk<R>(0, 0);
        const int k0 = tri == 0 ? j : i + 1, k1 = tri == 0 ? i - 1 : j;
        for (int k = k0; k <= k1; ++k) {
            sb_stage_T(Xa, A, lda, n, R0 + i * SB_TB, R0 + k * SB_TB);
            sb_stage_M(Xb, D, k, j);
            __syncthreads();
            sb_mm64(Xa, Xb, acc);
            __syncthreads();
        }
        // S into Xb, inv(T_ii) into Xa; X_ij = -inv(T_ii) S
        {
            const int tr = threadIdx.x >> 4, tc = threadIdx.x & 15;
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) Xb[(tr + 16 * a) * (SB_TB + 1) + tc + 16 * b] = acc[a][b];
        }
        sb_stage_inv(Xa, inv64, 4 * q + i, tri);
        __syncthreads();
        C x[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) x[a][b] = mk<R>(0, 0);
        sb_mm64(Xa, Xb, x);
        sb_store_acc(D, i, j, x, (R)-1);
        __syncthreads();
    }
}

// K1_q, K2_q: the 64 x 64 output tile (it, jt) of D_q T[q rows, P columns], P the block one or two before q in
// solve order. Grid (16 tiles, ns, 4 = triangle x {K1, K2}).
template <typename R>
__global__ void __launch_bounds__(256) k_sb_couple(const cpx<R> *A, long lda, int n, int ns, cpx<R> *mats)
{
    typedef cpx<R> C;
    extern __shared__ __align__(16) unsigned char sbc_raw[];
    C *Xa = reinterpret_cast<C *>(sbc_raw), *Xb = Xa + SB_TB * (SB_TB + 1);
    const int it = blockIdx.x / 4, jt = blockIdx.x % 4, q = blockIdx.y, tri = blockIdx.z / 2, m = blockIdx.z % 2 + 1;
    const int pos = tri == 0 ? q : ns - 1 - q;
    C *K = sb_mat(mats, ns, tri, m, q);
    C acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = mk<R>(0, 0);
    if (pos >= m) {
        const int P = tri == 0 ? q - m : q + m;
        const C *D = sb_mat(mats, ns, tri, 0, q);
        const int k0 = tri == 0 ? 0 : it, k1 = tri == 0 ? it : 3;      // D_q is block lower / upper triangular
        for (int kt = k0; kt <= k1; ++kt) {
            sb_stage_M(Xa, D, it, kt);
            sb_stage_T(Xb, A, lda, n, q * SB + kt * SB_TB, P * SB + jt * SB_TB);
            __syncthreads();
            sb_mm64(Xa, Xb, acc);
            __syncthreads();
        }
    }
    sb_store_acc(K, it, jt, acc, (R)1);
}

// ---- the solve ------------------------------------------------------------------------------------------------------
template <typename R>
struct SbSolve {
    const cpx<R> *A; long lda; int n, ns, nch;
    const cpx<R> *dinv, *k1, *k2;      // this triangle's [ns][SB][SB]
    const cpx<R> *Tin; cpx<R> *Xout;   // right-hand sides and solution, n x nrhs row-major
    cpx<R> *Tx;                        // published running right-hand sides, n x SB_NR
    int nrhs, backward, vec16;
    int *yflag, *tflag;                // [nch]: chunk's y / t published in the call of this epoch
    const int *epoch_ptr; int *err;
};

// acc[c] += sum_{kk < 64} M[r][kk] X[kk][c], thread (r = tid / 16, h = tid % 16) taking kk = h, h + 16, ...; a batch
// of terms' shared-memory reads before their products
template <typename R>
__device__ __forceinline__ void sb_acc_tile(const cpx<R> *Mt, const cpx<R> *X, cpx<R> (&acc)[SB_NR])
{
    constexpr int XS = sb_xs<R>(), NK = SB_KT / SB_TPR;
    const int r = threadIdx.x / SB_TPR, h = threadIdx.x % SB_TPR;
    const cpx<R> *row = Mt + r * SB_TS;
    if constexpr (sizeof(R) == 4) {
        cpx<float> v[NK];
        float4 y[NK][SB_NR / 2];
#pragma unroll
        for (int u = 0; u < NK; ++u) {
            const int kk = h + SB_TPR * u;
            v[u] = row[kk];
            const float4 *x = reinterpret_cast<const float4 *>(X + (size_t)kk * XS);
#pragma unroll
            for (int c2 = 0; c2 < SB_NR / 2; ++c2) y[u][c2] = x[c2];
        }
#pragma unroll
        for (int u = 0; u < NK; ++u)
#pragma unroll
            for (int c2 = 0; c2 < SB_NR / 2; ++c2) {
                cfma<float>(acc[2 * c2], v[u], mk<float>(y[u][c2].x, y[u][c2].y));
                cfma<float>(acc[2 * c2 + 1], v[u], mk<float>(y[u][c2].z, y[u][c2].w));
            }
    } else {
        constexpr int U = 2;
#pragma unroll
        for (int i0 = 0; i0 < NK; i0 += U) {
            cpx<double> v[U];
            double2 y[U][SB_NR];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int kk = h + SB_TPR * (i0 + u);
                v[u] = row[kk];
                const double2 *x = reinterpret_cast<const double2 *>(X + (size_t)kk * XS);
#pragma unroll
                for (int c = 0; c < SB_NR; ++c) y[u][c] = x[c];
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int c = 0; c < SB_NR; ++c) cfma<double>(acc[c], v[u], mk<double>(y[u][c].x, y[u][c].y));
        }
    }
}

// the 16 lanes of a chunk row: a halving exchange (4 + 2 + 1 values) leaves lane h with the sum of column h / 2
// over 8 lanes, the last exchange adds its partner's (lanes h and h ^ 1 hold the same column)
template <typename R>
__device__ __forceinline__ cpx<R> sb_reduce_scatter(cpx<R> (&acc)[SB_NR])
{
    const int h = threadIdx.x % SB_TPR;
    cpx<R> a4[4], a2[2];
    const bool hi8 = h & 8, hi4 = h & 4, hi2 = h & 2;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const cpx<R> send = hi8 ? acc[j] : acc[j + 4], keep = hi8 ? acc[j + 4] : acc[j];
        a4[j] = mk<R>(keep.x + __shfl_xor_sync(0xffffffffu, send.x, 8), keep.y + __shfl_xor_sync(0xffffffffu, send.y, 8));
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const cpx<R> send = hi4 ? a4[j] : a4[j + 2], keep = hi4 ? a4[j + 2] : a4[j];
        a2[j] = mk<R>(keep.x + __shfl_xor_sync(0xffffffffu, send.x, 4), keep.y + __shfl_xor_sync(0xffffffffu, send.y, 4));
    }
    const cpx<R> send = hi2 ? a2[0] : a2[1], keep = hi2 ? a2[1] : a2[0];
    const cpx<R> a1 = mk<R>(keep.x + __shfl_xor_sync(0xffffffffu, send.x, 2), keep.y + __shfl_xor_sync(0xffffffffu, send.y, 2));
    return mk<R>(a1.x + __shfl_xor_sync(0xffffffffu, a1.x, 1), a1.y + __shfl_xor_sync(0xffffffffu, a1.y, 1));
}

// waits (threads 0 .. cnt-1, one flag each) until flags[c0 ..] carry epoch; false (and M25_DEV_TIMEOUT) after about
// 2^21 polls or once another CTA has reported an error
__device__ __forceinline__ bool sb_wait_flags(const int *flags, int c0, int cnt, int epoch, int *err, int *ok)
{
    if ((int)threadIdx.x < cnt) {
        long it = 0;
        while ((int)ld_acquire_u32((const unsigned *)(flags + c0 + threadIdx.x)) != epoch) {
            if ((++it & 1023) == 0 && (it > (1L << 21) || *(volatile int *)err)) {
                *ok = 0;
                dev_error(err, M25_DEV_TIMEOUT);
                break;
            }
        }
    }
    __syncthreads();
    return *ok != 0;
}

// NBUF: tiles in the ring; TPB: tiles a product waits for at once (1, or a whole task of 4 with NBUF = 8)
template <typename R, int NBUF, int TPB>
__global__ void __launch_bounds__(SB_NT, 1) k_trsv_sb(SbSolve<R> a)
{
    static_assert(SB_KTS % TPB == 0 && NBUF >= 2 * TPB, "whole batches, one in flight beside the one in use");
    typedef cpx<R> C;
    constexpr int XS = sb_xs<R>();
    extern __shared__ __align__(16) unsigned char sb_raw[];
    C *tiles = reinterpret_cast<C *>(sb_raw);                        // [NBUF][SBC][SB_TS]
    C *Xs = tiles + (size_t)NBUF * SBC * SB_TS;                     // [SB][XS]: y_s, or the t of a block (phase 4)
    C *slots = Xs + (size_t)SB * XS;                                // [SB_CHMAX][SBC][SB_NR]
    __shared__ int ok;
    const int G = gridDim.x, g = blockIdx.x, tid = threadIdx.x;
    const int n = a.n, ns = a.ns, nch = a.nch, nrhs = a.nrhs;
    // roles: CTAs g < SB_GA take the chain's products (y, u, w) of chunks c = g + k SB_GA (chunk c % 8 of every
    // third block: one live chunk at a time); the others hold the running right-hand sides of chunks
    // c = g - SB_GA + k (G - SB_GA) and update them
    const bool chain = g < SB_GA;
    const int idx = chain ? g : g - SB_GA, stride = chain ? SB_GA : G - SB_GA;
    const int nmine = idx < nch ? (nch - 1 - idx) / stride + 1 : 0;
    if (nmine == 0) return;
    const int epoch = *(volatile const int *)a.epoch_ptr;
    auto chunk_of = [&](int k) { return idx + k * stride; };
    auto slot_of = [&](int k) { return chain ? (k & 1) : k; };
    auto q_of_pos = [&](int p) { return a.backward ? ns - 1 - p : p; };
    auto pos_k = [&](int k) { const int q = chunk_of(k) / SB_CPB; return a.backward ? ns - 1 - q : q; };
    int pmax = 0;
    for (int k = 0; k < nmine; ++k) pmax = max(pmax, pos_k(k));
    const int s_last = chain ? pmax - 1 : pmax - 3;
    // ---- the task order (every CTA's loader and products follow it): a task is (step s, phase ph, chunk k) ---------
    // chain CTAs: for each of their chunks in position order (position p), w at step max(p - 3, -1), u at p - 2
    // (p >= 2), y at p - 1 (p >= 1). Updating CTAs: at each step s, their chunks at positions >= s + 3 in position
    // order (the one at s + 3 first: its t is published). Both O(1) a task.
    struct Cur { int s, ph, k, j, t, jlo; bool done; };
    auto kj = [&](int j) { return a.backward ? nmine - 1 - j : j; };        // my j-th chunk by position
    auto posj = [&](int j) { return pos_k(kj(j)); };
    auto settle = [&](Cur &c) {                      // from (j, t) / (s, j): the task, or done
        if (chain) {
            for (;;) {
                if (c.j >= nmine) { c.done = true; return; }
                const int p = posj(c.j);
                if (c.t == 0) { c.s = max(p - 3, -1); c.ph = 4; break; }
                if (c.t == 1 && p >= 2) { c.s = p - 2; c.ph = 1; break; }
                if (c.t == 2 && p >= 1) { c.s = p - 1; c.ph = 0; break; }
                if (++c.t > 2) { c.t = 0; ++c.j; }
            }
        } else {
            if (c.j >= nmine) {
                if (++c.s > s_last) { c.done = true; return; }
                while (posj(c.jlo) < c.s + 3) ++c.jlo;
                c.j = c.jlo;
            }
            c.ph = posj(c.j) == c.s + 3 ? 2 : 3;
        }
        c.k = kj(c.j);
    };
    auto first = [&](Cur &c) {
        c.done = false; c.j = 0; c.t = 0; c.s = 0; c.jlo = 0;
        if (!chain) {
            if (s_last < 0) { c.done = true; return; }
            while (c.jlo < nmine && posj(c.jlo) < 3) ++c.jlo;
            c.j = c.jlo;
        }
        settle(c);
    };
    auto next = [&](Cur &c) {
        if (chain) { if (++c.t > 2) { c.t = 0; ++c.j; } }
        else ++c.j;
        settle(c);
    };
    // ---- the tile ring: the loader's cursor runs NBUF - 1 tiles ahead of the products -------------------------------
    Cur lc;
    int lkt = -1, issued = 0;
    const C *lsrc = nullptr;                         // the loader's task: its matrix rows, stride, valid extent
    long lld = SB;
    int lrv = SBC, lcv = SB, lv16 = 1;
    first(lc);
    auto load_task = [&]() {
        const int c = chunk_of(lc.k), q = c / SB_CPB;
        if (lc.ph == 2 || lc.ph == 3) {                                  // the factor: the chunk's rows, block s columns
            const int c0 = q_of_pos(lc.s) * SB;
            lsrc = a.A + (size_t)c * SBC * a.lda + c0;
            lld = a.lda;
            lrv = min(SBC, n - c * SBC);
            lcv = min(SB, n - c0);
            lv16 = a.vec16;
        } else {                                                         // K1, K2 or D: the chunk's rows of block q
            const C *m = lc.ph == 0 ? a.k1 : lc.ph == 1 ? a.k2 : a.dinv;
            lsrc = m + ((size_t)q * SB + (c % SB_CPB) * SBC) * SB;
            lld = SB;
            lrv = SBC;
            lcv = SB;
            lv16 = 1;
        }
    };
    if (!lc.done) load_task();
    auto issue = [&]() {
        if (!lc.done && ++lkt >= SB_KTS) {
            lkt = 0;
            next(lc);
            if (!lc.done) load_task();
        }
        if (!lc.done) {
            C *dst = tiles + (size_t)(issued % NBUF) * SBC * SB_TS;
            const C *src = lsrc + lkt * SB_KT;
            const long ld = lld;
            const int rv = lrv, cv = lcv - lkt * SB_KT;
            const bool v16 = lv16;
            if constexpr (sizeof(R) == 4) {
                if (v16) {                                            // 16-byte pieces: two entries
#pragma unroll
                    for (int i = 0; i < SBC * SB_KT / 2 / SB_NT; ++i) {
                        const int p = tid + SB_NT * i, r = p / (SB_KT / 2), e = 2 * (p % (SB_KT / 2));
                        C *d = dst + (size_t)r * SB_TS + e;
                        if (r < rv && e + 1 < cv) sb_cp16(d, src + (size_t)r * ld + e);
                        else {
                            d[1] = mk<R>(0, 0);
                            if (r < rv && e < cv) sb_cp8(d, src + (size_t)r * ld + e);
                            else d[0] = mk<R>(0, 0);
                        }
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < SBC * SB_KT / SB_NT; ++i) {
                        const int p = tid + SB_NT * i, r = p / SB_KT, e = p % SB_KT;
                        C *d = dst + (size_t)r * SB_TS + e;
                        if (r < rv && e < cv) sb_cp8(d, src + (size_t)r * ld + e);
                        else *d = mk<R>(0, 0);
                    }
                }
            } else {
#pragma unroll
                for (int i = 0; i < SBC * SB_KT / SB_NT; ++i) {
                    const int p = tid + SB_NT * i, r = p / SB_KT, e = p % SB_KT;
                    C *d = dst + (size_t)r * SB_TS + e;
                    if (r < rv && e < cv) sb_cp16(d, src + (size_t)r * ld + e);
                    else *d = mk<R>(0, 0);
                }
            }
            ++issued;
        }
        sb_commit();                                                  // (an empty group past the last tile)
    };
    // ---- the running right-hand sides of my chunks: b (the updating CTAs) ---------------------------------------------
    if (!chain)
        for (int e = tid; e < nmine * SBC * SB_NR; e += SB_NT) {
            const int k = e / (SBC * SB_NR), r = (e / SB_NR) % SBC, cc = e % SB_NR, row = chunk_of(k) * SBC + r;
            slots[e] = (row < n && cc < nrhs) ? a.Tin[(size_t)row * nrhs + cc] : mk<R>(0, 0);
        }
    if (tid == 0) ok = 1;
    for (int i = 0; i < NBUF - TPB; ++i) issue();
    __syncthreads();
    // one staged vector of SB rows: from src (row stride ld, columns < cols), rows past n and columns past cols zero;
    // every load before any store
    auto stage = [&](const C *src, int ld, int cols, int row0) {
        C v[SB * SB_NR / SB_NT];
#pragma unroll
        for (int i = 0; i < SB * SB_NR / SB_NT; ++i) {
            const int e = tid + SB_NT * i, r = e / SB_NR, cc = e % SB_NR, row = row0 + r;
            if (row < n && cc < cols) {
                typedef typename vec2_of<R>::type V2;
                const V2 w = __ldcg(reinterpret_cast<const V2 *>(src) + (size_t)row * ld + cc);
                v[i] = mk<R>(w.x, w.y);
            } else {
                v[i] = mk<R>(0, 0);
            }
        }
#pragma unroll
        for (int i = 0; i < SB * SB_NR / SB_NT; ++i) {
            const int e = tid + SB_NT * i;
            Xs[(e / SB_NR) * XS + e % SB_NR] = v[i];
        }
        __syncthreads();
    };
    // a chunk's slot out: y into the solution (columns < nrhs) or t into Tx; then the chunk's flag
    auto publish = [&](int k, bool is_y) {
        const int c = chunk_of(k), r = tid / SB_NR, cc = tid % SB_NR, row = c * SBC + r;
        if (tid < SBC * SB_NR && row < n) {
            const C v = slots[(size_t)slot_of(k) * SBC * SB_NR + tid];
            if (is_y) { if (cc < nrhs) a.Xout[(size_t)row * nrhs + cc] = v; }
            else a.Tx[(size_t)row * SB_NR + cc] = v;
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            atomicExch((is_y ? a.yflag : a.tflag) + c, epoch);
        }
    };
    int used = 0, cur = -2;
    Cur cc;
    for (first(cc); !cc.done; next(cc)) {
        const int s = cc.s, ph = cc.ph, k = cc.k;
        if (s != cur) {                                               // a new step: y_s of the block at position s
            cur = s;
            if (s >= 0) {
                const int q = q_of_pos(s), c0 = q * SB_CPB, cnt = min(SB_CPB, nch - c0);
                if (!sb_wait_flags(a.yflag, c0, cnt, epoch, a.err, &ok)) { sb_wait_group<0>(); return; }
                stage(a.Xout, nrhs, nrhs, q * SB);
            }
        }
        if (ph == 4) {                                                // w: the t of the whole block
            if (s < 0) {
                stage(a.Tin, nrhs, nrhs, q_of_pos(pos_k(k)) * SB);
            } else {
                const int q = q_of_pos(s + 3), c0 = q * SB_CPB, cnt = min(SB_CPB, nch - c0);
                if (!sb_wait_flags(a.tflag, c0, cnt, epoch, a.err, &ok)) { sb_wait_group<0>(); return; }
                stage(a.Tx, SB_NR, SB_NR, q * SB);
            }
        }
        C acc[SB_NR];
#pragma unroll
        for (int j = 0; j < SB_NR; ++j) acc[j] = mk<R>(0, 0);
        for (int kt0 = 0; kt0 < SB_KTS; kt0 += TPB) {
#pragma unroll
            for (int i = 0; i < TPB; ++i) issue();
            sb_wait_group<NBUF - TPB>();                              // this batch's copies have landed
            __syncthreads();
#pragma unroll
            for (int i = 0; i < TPB; ++i) {
                sb_acc_tile<R>(tiles + (size_t)(used % NBUF) * SBC * SB_TS, Xs + (size_t)(kt0 + i) * SB_KT * XS, acc);
                ++used;
            }
            __syncthreads();                                          // (the buffers are the next copies')
        }
        const C v = sb_reduce_scatter<R>(acc);
        if (!(tid & 1)) {                                             // lanes h, h ^ 1 hold column h / 2
            C *sl = slots + (size_t)slot_of(k) * SBC * SB_NR + (tid / SB_TPR) * SB_NR + (tid % SB_TPR) / 2;
            if (ph == 4) *sl = v;
            else *sl -= v;
        }
        __syncthreads();
        if (ph == 0 || (s < 0 && pos_k(k) == 0)) publish(k, true);
        else if (ph == 2) publish(k, false);
    }
    sb_wait_group<0>();
}

// ---- host -----------------------------------------------------------------------------------------------------------
static int sb_sms()
{
    int dev, sms;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    return sms;
}

// Whether the solves of a factor of size n take this form: n >= SB_MIN_N and a CTA's chunks within SB_CHMAX, for
// complex64 and complex128 factors; M25_TRSV=pipe keeps the 64-row-block solves everywhere, M25_TRSV=c64 keeps them
// for complex128 factors.
bool m25_sb_enabled(int n, int single)
{
    static const int on = [] {
        const char *e = getenv("M25_TRSV");
        return (e && !strcmp(e, "pipe")) ? 0 : (e && !strcmp(e, "c64")) ? 1 : 2;
    }();
    if (!on || (!single && on < 2) || n < SB_MIN_N) return false;
    const int GB = sb_sms() - SB_GA, nch = (n + SBC - 1) / SBC;
    return GB > 0 && (nch + GB - 1) / GB <= SB_CHMAX;
}

template <typename R>
static size_t sb_layout(int n, size_t *off_tx, size_t *off_flags)
{
    const size_t ns = (n + SB - 1) / SB, nch = (n + SBC - 1) / SBC;
    size_t o = 2 * 3 * ns * SB * SB * sizeof(cpx<R>);
    o = (o + 255) / 256 * 256;
    *off_tx = o;
    o += (size_t)n * SB_NR * sizeof(cpx<R>);
    o = (o + 255) / 256 * 256;
    *off_flags = o;
    o += 4 * nch * sizeof(int);
    return (o + 255) / 256 * 256;
}

size_t m25_sb_bytes(int n, int single)
{
    if (!m25_sb_enabled(n, single)) return 0;
    size_t a, b;
    return single ? sb_layout<float>(n, &a, &b) : sb_layout<double>(n, &a, &b);
}

template <typename R>
static int sb_prepare_impl(const cpx<R> *A, long lda, int n, const cpx<R> *inv64, unsigned char *sb, cudaStream_t s)
{
    size_t otx, ofl;
    sb_layout<R>(n, &otx, &ofl);
    const int ns = (n + SB - 1) / SB, nch = (n + SBC - 1) / SBC;
    cpx<R> *mats = reinterpret_cast<cpx<R> *>(sb);
    const size_t sm = 2 * sizeof(cpx<R>) * SB_TB * (SB_TB + 1);
    M25_CHECK(cudaFuncSetAttribute(k_sb_dinv<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    M25_CHECK(cudaFuncSetAttribute(k_sb_couple<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_sb_dinv<R><<<dim3(4, ns, 2), 256, sm, s>>>(A, lda, n, ns, inv64, mats);
    M25_LAUNCH_CHECK("k_sb_dinv");
    k_sb_couple<R><<<dim3(16, ns, 4), 256, sm, s>>>(A, lda, n, ns, mats);
    M25_LAUNCH_CHECK("k_sb_couple");
    M25_CHECK(cudaMemsetAsync(sb + ofl, 0, 4 * (size_t)nch * sizeof(int), s));
    return M25_OK;
}

// D, K1, K2 of both triangles of the factor A (inv64: the 64-row diagonal-block inverses of k_block_inverses) into
// sb (m25_sb_bytes), and the solves' flags zeroed
int m25_sb_prepare(const void *A, long lda, int n, int single, const void *inv64, void *sb, cudaStream_t s)
{
    return single ? sb_prepare_impl<float>((const cpx<float> *)A, lda, n, (const cpx<float> *)inv64,
                                           (unsigned char *)sb, s)
                  : sb_prepare_impl<double>((const cpx<double> *)A, lda, n, (const cpx<double> *)inv64,
                                            (unsigned char *)sb, s);
}

template <typename R>
static int sb_solve_impl(const cpx<R> *A, long lda, int n, unsigned char *sb, const cpx<R> *Tin, cpx<R> *Xout,
                         int nrhs, int backward, const int *epoch, int *err, cudaStream_t s)
{
    size_t otx, ofl;
    sb_layout<R>(n, &otx, &ofl);
    const int ns = (n + SB - 1) / SB, nch = (n + SBC - 1) / SBC;
    const int G = std::min(sb_sms(), SB_GA + nch);
    M25_REQUIRE(G > SB_GA && (nch + G - SB_GA - 1) / (G - SB_GA) <= SB_CHMAX,
                "m25_sb_solve: n too large for the 256-row-block solve");
    M25_REQUIRE(nrhs >= 1 && nrhs <= SB_NR, "m25_sb_solve: 1 to 8 right-hand sides");
    cpx<R> *mats = reinterpret_cast<cpx<R> *>(sb);
    int *flags = reinterpret_cast<int *>(sb + ofl);
    const int tri = backward ? 1 : 0;
    SbSolve<R> args{A, lda, n, ns, nch,
                    sb_mat(mats, ns, tri, 0, 0), sb_mat(mats, ns, tri, 1, 0), sb_mat(mats, ns, tri, 2, 0),
                    Tin, Xout, reinterpret_cast<cpx<R> *>(sb + otx), nrhs, backward,
                    (int)((lda % 2 == 0) && (reinterpret_cast<uintptr_t>(A) % 16 == 0)),
                    flags + (size_t)tri * 2 * nch, flags + (size_t)tri * 2 * nch + nch, epoch, err};
    // the tile ring: complex64, 8 tiles whose products wait for a task's 4 tiles at once (two barriers a task instead
    // of eight: 1.94 against 2.07 ms a pair at N = 18,788); M25_SB_TPB=1 waits for one tile at a time in a ring of
    // M25_SB_NBUF=3|5|8 (default 5; the depth alone measured the same). complex128 takes 3 single tiles, its tiles
    // being twice as large
    static const int want = [] { const char *e = getenv("M25_SB_NBUF"); return e ? atoi(e) : 5; }();
    static const int tpb = [] { const char *e = getenv("M25_SB_TPB"); return e ? atoi(e) : 4; }();
    int optin = 0, dev = 0;
    M25_CHECK(cudaGetDevice(&dev));
    M25_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    int nbuf = want >= 8 ? 8 : want >= 5 ? 5 : 3;
    const bool batch4 = sizeof(R) == 4 && tpb == 4 && sb_smem<R>(8) <= (size_t)optin;
    if (batch4) nbuf = 8;
    while (nbuf > 3 && sb_smem<R>(nbuf) > (size_t)optin) nbuf = nbuf == 8 ? 5 : 3;
    const size_t sm = sb_smem<R>(nbuf);
    M25_REQUIRE(sm <= (size_t)optin, "m25_sb_solve: shared memory");
    const void *kf = batch4 ? (const void *)k_trsv_sb<R, 8, 4>
                   : nbuf == 8 ? (const void *)k_trsv_sb<R, 8, 1> : nbuf == 5 ? (const void *)k_trsv_sb<R, 5, 1>
                                                                         : (const void *)k_trsv_sb<R, 3, 1>;
    M25_CHECK(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    void *kargs[] = {&args};
    M25_CHECK(cudaLaunchCooperativeKernel(kf, dim3(G), dim3(SB_NT), kargs, sm, s));
    m25_note_launch();
    return M25_OK;
}

// One triangle of the solve (backward 0: U^T y = Tin; 1: L^T z = Tin) into Xout (n x nrhs, nrhs <= 8), with the
// data of m25_sb_prepare; flags compared with *epoch, which the caller bumps once per pair of solves
int m25_sb_solve(const void *A, long lda, int n, int single, void *sb, const void *Tin, void *Xout, int nrhs,
                 int backward, const int *epoch, int *err, cudaStream_t s)
{
    return single ? sb_solve_impl<float>((const cpx<float> *)A, lda, n, (unsigned char *)sb, (const cpx<float> *)Tin,
                                         (cpx<float> *)Xout, nrhs, backward, epoch, err, s)
                  : sb_solve_impl<double>((const cpx<double> *)A, lda, n, (unsigned char *)sb,
                                          (const cpx<double> *)Tin, (cpx<double> *)Xout, nrhs, backward, epoch, err, s);
}
