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
#include <type_traits>
#include <algorithm>
#include <mutex>

#include "common.cuh"

static inline cudaStream_t S(void *s) { return (cudaStream_t)s; }
int *m25_dev_err_word();
int m25_check_dev_err(cudaStream_t s, const char *what);
int m25_umma_trailing(float *A, long lda, int M, int Ncol, int K, const float *L21, const float *U12, void *work,
                      size_t work_bytes, cudaStream_t s);
size_t m25_umma_workspace(int n, int nb);

#define NB 64
#define NB2 256
#define PANEL_THREADS 256
static_assert(PANEL_THREADS >= 2 * NB, "the panel's row copies take a thread a column for two rows");

struct PanelWork {
    double *cand_val;     // [2][G]
    int *cand_idx;        // [2][G]
    double *cand_row;     // [2][G][NB] complex (as R pairs; sized for double)
    double *drow;         // [2][NB] complex
    GridBarrier bar;
    unsigned *gen;        // [2][G]
    unsigned long long *ll_cand;   // [2][G][LL_REC] flagged words: a block's candidate |re| + |im| and row
    unsigned long long *ll_row;    // [2][G][4 NB]: its candidate row
    unsigned long long *ll_drow;   // [2][4 NB]: the diagonal row
};

// The panel's exchange records: 64-bit words of a 32-bit payload and a 32-bit flag (the column + 1 it belongs
// to), written and read whole (a naturally aligned 64-bit access is single-copy atomic), so that a reader that
// sees the flag sees the payload: no fence, no separate ready flag, one round trip to L2 per exchange.
__device__ __forceinline__ void ll_put(unsigned long long *p, unsigned payload, unsigned flag)
{
    const unsigned long long w = ((unsigned long long)flag << 32) | payload;
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(w) : "memory");
}
__device__ __forceinline__ unsigned long long ll_get(const unsigned long long *p)
{
    unsigned long long w;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
    return w;
}
// waits until the K words p[0], p[stride], ... carry flag; their payloads in out. Bounded: false after about 2^22
// polls or once another block has reported an error.
template <int K>
__device__ __forceinline__ bool ll_wait(const unsigned long long *p, int stride, unsigned flag, unsigned *out,
                                        const int *err)
{
    long it = 0;
    for (;;) {
        bool all = true;
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const unsigned long long w = ll_get(p + (size_t)q * stride);
            out[q] = (unsigned)w;
            all = all && (unsigned)(w >> 32) == flag;
        }
        if (all) return true;
        if ((++it & 1023) == 0 && (it > (1L << 22) || *(volatile const int *)err)) return false;
    }
}


// The same exchange inside a thread-block cluster: each block's records in its own shared memory, written there and
// read by the other blocks of the cluster through distributed shared memory (generic addresses of their shared
// memory), at cluster scope; polled the same bounded way.
__device__ __forceinline__ void cl_put(unsigned long long *p, unsigned payload, unsigned flag)
{
    const unsigned long long w = ((unsigned long long)flag << 32) | payload;
    asm volatile("st.relaxed.cluster.u64 [%0], %1;" ::"l"(p), "l"(w) : "memory");
}
__device__ __forceinline__ unsigned long long cl_get(const unsigned long long *p)
{
    unsigned long long w;
    asm volatile("ld.relaxed.cluster.u64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
    return w;
}
template <bool CL>
__device__ __forceinline__ void x_put(unsigned long long *p, unsigned payload, unsigned flag)
{
    if (CL) cl_put(p, payload, flag);
    else ll_put(p, payload, flag);
}
template <int K, bool CL>
__device__ __forceinline__ bool x_wait(const unsigned long long *p, int stride, unsigned flag, unsigned *out,
                                       const int *err)
{
    if (!CL) return ll_wait<K>(p, stride, flag, out, err);
    long it = 0;
    for (;;) {
        bool all = true;
#pragma unroll
        for (int q = 0; q < K; ++q) {
            const unsigned long long w = cl_get(p + (size_t)q * stride);
            out[q] = (unsigned)w;
            all = all && (unsigned)(w >> 32) == flag;
        }
        if (all) return true;
        if ((++it & 1023) == 0 && (it > (1L << 22) || *(volatile const int *)err)) return false;
    }
}

#define PANEL_NONE 0x7fffffff
#define LL_REC 32             // words a candidate record (256 bytes: polled by every block, one record a line pair)
// a cluster panel's records, after its rows in shared memory
struct PanelRecords {
    unsigned long long cand[2][LL_REC];
    unsigned long long row[2][4 * NB];
    unsigned long long drow[2][4 * NB];
};

// The largest |re| + |im| and its row over a warp (the first row on ties: izamax / icamax)
template <typename R>
__device__ __forceinline__ void warp_argmax(R &v, int &row)
{
    for (int o = 16; o; o >>= 1) {
        const R ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int orow = __shfl_xor_sync(0xffffffffu, row, o);
        if (ov > v || (ov == v && orow < row)) { v = ov; row = orow; }
    }
}

// The panel (GEPP over jb <= NB columns k0 .., rows k0 .. n) with each block's rows in shared memory for the whole
// panel (Ps[c * cs + i] is row r0 + i, column k0 + c): global memory is read once and written once. Per column j:
// (1) the block's candidate; (2) warp 0 brings the candidate row and the diagonal row (where the block holds it) up
// to date and publishes them with the candidate; (3) the deferred part of the update (below), run while the
// exchange is in flight; (4) every block's candidate read and reduced; (5) the pivot row and the diagonal row (from
// the block's own shared memory where it holds them); (6) the interchange, the scaling of column j and the update
// of column j + 1 only, which yields the next candidates. Two round trips to L2 and three block barriers a column.
//
// The updates are grouped by GRP columns so that the columns past the current group are read and written once a
// group rather than once a column (the rank-1 updates made the panel bound by shared-memory bandwidth): within the
// group [g0, gend) a column's update reaches only the group's own later columns; at the next group's first column,
// step (3) applies the whole group's GRP terms to every column past it (and step 6 of the group's last column to
// the column after it, which is searched next). A row published as a candidate goes out in full (the group's terms
// due on the columns past the group added on the way, not stored), the diagonal row as stored (it moves into
// another block's rows, where those terms are still applied). Every entry still takes its terms a -= l U one at a
// time in column order: the results are those of the column-by-column order.
//
// CL: the panel's blocks are one thread-block cluster (a panel of up to 16 blocks' rows) and the exchange goes
// through distributed shared memory instead of L2: the same records and bounded polls, each block's records after
// its rows in its own shared memory (zeroed, then a cluster barrier, before the first column; a cluster barrier
// before any block leaves, so that no block reads the shared memory of one that has). The other blocks' records
// are a few hundred cycles away instead of an L2 round trip, which the trailing update's traffic makes long.
#define GRP 8
// the block's candidate from the warps' ones (sv, si of nw warps): one butterfly in every warp
template <typename R>
__device__ __forceinline__ void block_argmax(R &v, int &row, const R *sv, const int *si, int lane, int nw)
{
    v = lane < nw ? sv[lane] : (R)-1;
    row = lane < nw ? si[lane] : PANEL_NONE;
    warp_argmax(v, row);
}
template <typename R, bool CL>
__global__ void __launch_bounds__(PANEL_THREADS) k_panel_smem(R *A, long lda, int n, int k0, int jb, int *ipiv,
                                                              PanelWork pw, int *err)
{
    typedef cpx<R> C;
    constexpr int WPC = sizeof(C) / 4;                    // 32-bit words a complex number
    constexpr int VW = sizeof(R) / 4;                     // 32-bit words of |re| + |im|
    constexpr int NWARP = PANEL_THREADS / 32;
    extern __shared__ unsigned char panel_raw[];
    C *Ps = reinterpret_cast<C *>(panel_raw);
    const unsigned *P32 = reinterpret_cast<const unsigned *>(Ps);
    const int G = gridDim.x, b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int rows = n - k0;
    const int cs = (rows + G - 1) / G;
    const int r0 = k0 + b * cs, r1 = min(n, r0 + cs);
    const int nr = max(0, r1 - r0);
    const int PW = jb * WPC;                              // payload words of one panel row
    PanelRecords *RX = reinterpret_cast<PanelRecords *>(panel_raw + ((size_t)cs * jb * sizeof(C) + 15) / 16 * 16);
    __shared__ __align__(16) C U[NB], D[NB], W[NB];       // pivot row, diagonal row, this block's published row
    __shared__ __align__(16) C Ug[GRP][NB];               // the current group's pivot rows
    __shared__ R sv[NWARP], sv2[NWARP];
    __shared__ int si[NWARP], si2[NWARP], sw2[NWARP];
    __shared__ int s_fail;
    for (int e = tid; e < nr * jb; e += PANEL_THREADS) {
        int c = e / nr, i = e % nr;
        Ps[c * cs + i] = ldc<R>(A, (size_t)(k0 + c) * lda + r0 + i);
    }
    if (tid == 0) s_fail = 0;
    if constexpr (CL) {
        unsigned long long *rz = reinterpret_cast<unsigned long long *>(RX);
        for (int e = tid; e < (int)(sizeof(PanelRecords) / 8); e += PANEL_THREADS) rz[e] = 0ull;
        __syncthreads();
        cooperative_groups::this_cluster().sync();
    }
    __syncthreads();
    R best = -1;                                          // this thread's candidate for column 0
    int bi = PANEL_NONE;
    for (int i = tid; i < nr; i += PANEL_THREADS) {
        const R v = abs1(Ps[i]);
        if (v > best) { best = v; bi = r0 + i; }
    }
    for (int j = 0; j < jb; ++j) {
        const int col = k0 + j, par = j & 1;
        const unsigned flag = (unsigned)col + 1u;
        const bool own_col = col >= r0 && col < r1;
        // this column's records: where this block publishes, and where block q's are read
        unsigned long long *my_rec, *my_row, *my_drow;
        if constexpr (CL) {
            my_rec = RX->cand[par]; my_row = RX->row[par]; my_drow = RX->drow[par];
        } else {
            my_rec = pw.ll_cand + ((size_t)par * G + b) * LL_REC;
            my_row = pw.ll_row + ((size_t)par * G + b) * (4 * NB);
            my_drow = pw.ll_drow + (size_t)par * (4 * NB);
        }
        auto rec_of = [&](int q, int which) -> const unsigned long long * {   // which: 0 record, 1 row, 2 diagonal
            if constexpr (CL) {
                unsigned long long *mine = which == 0 ? RX->cand[par] : which == 1 ? RX->row[par] : RX->drow[par];
                return cooperative_groups::this_cluster().map_shared_rank(mine, (unsigned)q);
            } else {
                return which == 0 ? pw.ll_cand + ((size_t)par * G + q) * LL_REC
                     : which == 1 ? pw.ll_row + ((size_t)par * G + q) * (4 * NB) : pw.ll_drow + (size_t)par * (4 * NB);
            }
        };
        const int g0 = j - j % GRP, gend = min(g0 + GRP, jb);
        const bool gstart = j > 0 && j == g0;             // the previous group's terms are due past column j
        const int pg0 = g0 - GRP;
        // (1) the block's candidate
        warp_argmax(best, bi);
        if (lane == 0) { sv[wid] = best; si[wid] = bi; }
        __syncthreads();                                  // (column j is complete for every row >= col)
        block_argmax(best, bi, sv, si, lane, NWARP);
        const int ec = own_col ? col - r0 : -1;                          // rows brought up to date eagerly
        const int eb = (bi != PANEL_NONE && bi != col) ? bi - r0 : -1;
        const int ep = bi != PANEL_NONE ? bi - r0 : -1;                  // the candidate's row (ec if bi == col)
        // (2) warp 0: the deferred update of those rows (as step 3 does it for the others), then the block's record
        if (wid == 0) {
            if (j > 0) {
                for (int q = 0; q < 2; ++q) {
                    const int e = q ? eb : ec;
                    if (e < 0) continue;
                    if (gstart) {
                        C lr[GRP];
#pragma unroll
                        for (int s = 0; s < GRP; ++s) lr[s] = Ps[(pg0 + s) * cs + e];
                        for (int c = j + 1 + lane; c < jb; c += 32) {
                            C a = Ps[c * cs + e];
#pragma unroll
                            for (int s = 0; s < GRP; ++s) cfms<R>(a, lr[s], Ug[s][c]);
                            Ps[c * cs + e] = a;
                        }
                    } else {
                        const C lp = Ps[(j - 1) * cs + e];
                        for (int c = j + 1 + lane; c < gend; c += 32) {
                            C a = Ps[c * cs + e];
                            cfms<R>(a, lp, U[c]);
                            Ps[c * cs + e] = a;
                        }
                    }
                }
                __syncwarp();
            }
            unsigned long long *rec = my_rec;
            if (lane == 0) {
                const unsigned *bv32 = reinterpret_cast<const unsigned *>(&best);
#pragma unroll
                for (int q = 0; q < VW; ++q) x_put<CL>(rec + q, bv32[q], flag);
                x_put<CL>(rec + VW, (unsigned)bi, flag);
            }
            unsigned long long *rrow = my_row;
            unsigned long long *drow = my_drow;
            for (int c = lane; c < jb; c += 32) {
                if (ep >= 0) {                             // the candidate row in full
                    C a = Ps[c * cs + ep];
                    if (c >= gend)
                        for (int s = g0; s < j; ++s) cfms<R>(a, Ps[s * cs + ep], Ug[s - g0][c]);
                    W[c] = a;
                    const unsigned *a32 = reinterpret_cast<const unsigned *>(&a);
#pragma unroll
                    for (int q = 0; q < WPC; ++q) x_put<CL>(rrow + c * WPC + q, a32[q], flag);
                }
                if (own_col) {                             // the diagonal row as stored
                    const C d = Ps[c * cs + ec];
                    const unsigned *d32 = reinterpret_cast<const unsigned *>(&d);
#pragma unroll
                    for (int q = 0; q < WPC; ++q) x_put<CL>(drow + c * WPC + q, d32[q], flag);
                }
            }
            __syncwarp();
        }
        // (3) the deferred update for the other rows >= col
        if (gstart) {
            // the previous group's GRP terms on every column past j: a thread a row (a warp on consecutive rows),
            // its multipliers in registers, the group's pivot rows read as broadcasts
            for (int i = max(0, col - r0) + tid; i < nr; i += PANEL_THREADS) {
                if (i == ec || i == eb) continue;
                C lr[GRP];
#pragma unroll
                for (int s = 0; s < GRP; ++s) lr[s] = Ps[(pg0 + s) * cs + i];
#pragma unroll 2
                for (int c = j + 1; c < jb; ++c) {
                    C a = Ps[c * cs + i];
#pragma unroll
                    for (int s = 0; s < GRP; ++s) cfms<R>(a, lr[s], Ug[s][c]);
                    Ps[c * cs + i] = a;
                }
            }
        } else if (j > 0) {
            // the previous column's term on the group's columns past j: two threads a row (adjacent lanes),
            // columns j + 1 + sub, j + 3 + sub, ...
            const int sub = tid & 1;
            for (int i = max(0, col - r0) + (tid >> 1); i < nr; i += PANEL_THREADS / 2) {
                if (i == ec || i == eb) continue;
                const C lp = Ps[(j - 1) * cs + i];
                for (int c = j + 1 + sub; c < gend; c += 2) {
                    C a = Ps[c * cs + i];
                    cfms<R>(a, lp, U[c]);
                    Ps[c * cs + i] = a;
                }
            }
        }
        // (4) every block's candidate
        R bv = -1;
        int brow = PANEL_NONE, bw = -1;
        if (tid < G) {
            unsigned wv[VW + 1];
            if (!x_wait<VW + 1, CL>(rec_of(tid, 0), 1, flag, wv, err)) {
                s_fail = 1;
                dev_error(err, M25_DEV_TIMEOUT);
            } else if ((int)wv[VW] != PANEL_NONE) {
                R v;
                memcpy(&v, wv, sizeof(R));
                bv = v; brow = (int)wv[VW]; bw = tid;
            }
        }
        for (int o = 16; o; o >>= 1) {
            const R ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int orow = __shfl_xor_sync(0xffffffffu, brow, o), ow = __shfl_xor_sync(0xffffffffu, bw, o);
            if (ov > bv || (ov == bv && orow < brow)) { bv = ov; brow = orow; bw = ow; }
        }
        if (lane == 0) { sv2[wid] = bv; si2[wid] = brow; sw2[wid] = bw; }
        __syncthreads();                                  // (and the deferred update is complete)
        if (s_fail) goto finish;
        bv = lane < NWARP ? sv2[lane] : (R)-1;              // the block's reduction by one butterfly a warp
        brow = lane < NWARP ? si2[lane] : PANEL_NONE;
        bw = lane < NWARP ? sw2[lane] : -1;
        for (int o = 16; o; o >>= 1) {
            const R ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int orow = __shfl_xor_sync(0xffffffffu, brow, o), ow = __shfl_xor_sync(0xffffffffu, bw, o);
            if (ov > bv || (ov == bv && orow < brow)) { bv = ov; brow = orow; bw = ow; }
        }
        if (bw < 0 || bw >= G) {
            if (tid == 0) dev_error(err, M25_DEV_INDEX);
            goto finish;
        }
        const int p = brow;
        if (b == 0 && tid == 0) ipiv[col] = p;
        // (5) every block: U[j ..]; the block that holds row col: all of U; the block that holds row p: D. The
        // pivot row comes in full (from W where the block published it), the diagonal row as stored. U also goes
        // into the group's rows for the terms past the group
        if (tid < PW) {
            const int q = tid % WPC;
            const bool own_p = b == bw, need_u = own_col || tid >= j * WPC;
            unsigned u = 0, d = 0;
            bool ok = true;
            if (own_p) {
                u = reinterpret_cast<const unsigned *>(W)[tid];
                if (own_col) d = P32[((size_t)(tid / WPC) * cs + (col - r0)) * WPC + q];
                else ok = x_wait<1, CL>(rec_of((col - k0) / cs, 2) + tid, 0, flag, &d, err);
            } else if (need_u) {
                ok = x_wait<1, CL>(rec_of(bw, 1) + tid, 0, flag, &u, err);
            }
            if (!ok) {
                s_fail = 1;
                dev_error(err, M25_DEV_TIMEOUT);
            } else {
                if (own_p || need_u) {
                    reinterpret_cast<unsigned *>(U)[tid] = u;
                    reinterpret_cast<unsigned *>(Ug[j - g0])[tid] = u;
                }
                if (own_p) reinterpret_cast<unsigned *>(D)[tid] = d;
            }
        }
        __syncthreads();
        if (s_fail) goto finish;
        // (6) rows col and p interchanged (whole panel rows), column j scaled by 1 / pivot, column j + 1 updated
        // (the rest of this column's update is deferred to the next column's step 3); the next candidates
        const C piv = U[j];
        C rc;
        if (piv.x == 0 && piv.y == 0) {
            if (b == 0 && tid == 0) dev_error(err, M25_DEV_ZEROPIV);
            rc = mk<R>(0, 0);
        } else {
            rc = cdiv<R>(mk<R>(1, 0), piv);
        }
        // the interchanged rows' copies spread over the block (one thread copying a row alone would hold every
        // other block up at the next exchange); the thread of row p writes its columns j and j + 1 itself
        {
            const int e = tid % NB, half = tid / NB;
            if (e < jb) {
                if (half == 0 && own_col) Ps[e * cs + (col - r0)] = U[e];
                if (half == 1 && b == bw && p != col && e != j && e != j + 1) Ps[e * cs + (p - r0)] = D[e];
            }
        }
        // column j + 1: the group's last term here, or (the group's last column) every term of the group
        const bool gfin = j + 1 == gend && j + 1 < jb;
        best = -1; bi = PANEL_NONE;
        for (int i = max(0, col - r0) + tid; i < nr; i += PANEL_THREADS) {
            const int row = r0 + i;
            if (row == col) continue;
            const bool isp = row == p;
            const C l = (isp ? D[j] : Ps[j * cs + i]) * rc;
            Ps[j * cs + i] = l;
            if (j + 1 < jb) {
                C a = isp ? D[j + 1] : Ps[(j + 1) * cs + i];
                if (gfin)
                    for (int s = g0; s < j; ++s) cfms<R>(a, isp ? D[s] : Ps[s * cs + i], Ug[s - g0][j + 1]);
                cfms<R>(a, l, U[j + 1]);
                Ps[(j + 1) * cs + i] = a;
                const R v = abs1(a);
                if (v > best) { best = v; bi = row; }
            }
        }
    }
    __syncthreads();
    for (int e = tid; e < nr * jb; e += PANEL_THREADS) {
        int c = e / nr, i = e % nr;
        stc<R>(A, (size_t)(k0 + c) * lda + r0 + i, Ps[c * cs + i]);
    }
finish:
    if constexpr (CL) cooperative_groups::this_cluster().sync();   // (no block leaves while another may read it)
}

// The same with the rows in global memory (when a block's rows do not fit in shared memory).
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
        // 3. the pivot: the best candidate over the blocks, the smallest row on ties (one warp, loads in parallel,
        //    past L1: the other blocks wrote them)
        if (tid < 32) {
            double bv = -1.0;
            int bw = -1, brow = 0x7fffffff;
            for (unsigned w = tid; w < G; w += 32) {
                double v = __ldcg(pw.cand_val + par * G + w);
                int ri = __ldcg(pw.cand_idx + par * G + w);
                if (ri == 0x7fffffff) continue;
                if (v > bv || (v == bv && ri < brow)) { bv = v; bw = (int)w; brow = ri; }
            }
            for (int o = 16; o; o >>= 1) {
                double ov = __shfl_xor_sync(0xffffffffu, bv, o);
                int ow = __shfl_xor_sync(0xffffffffu, bw, o), orow = __shfl_xor_sync(0xffffffffu, brow, o);
                if (ov > bv || (ov == bv && orow < brow)) { bv = ov; bw = ow; brow = orow; }
            }
            if (tid == 0) {
                si[0] = bw;
                s_p = brow;
                if (b == 0 && bw >= 0) ipiv[col] = brow;
            }
        }
        __syncthreads();
        const int wb = si[0], p = s_p;
        if (wb < 0) { dev_error(err, M25_DEV_INDEX); return; }
        if (tid < jb) {           // other blocks' writes: read past L1, one load each
            typedef typename vec2_of<R>::type V2;
            const V2 u = __ldcg(reinterpret_cast<const V2 *>(cand_row + ((size_t)par * G + wb) * NB + tid));
            const V2 d = __ldcg(reinterpret_cast<const V2 *>(drow + par * NB + tid));
            U[tid] = mk<R>(u.x, u.y);
            D[tid] = mk<R>(d.x, d.y);
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

// ---- interchanges as one permutation ----------------------------------------------------------------------------
// The interchanges of rows r0 + i and p_i = ipiv[r0 + i], i = 0 .. nsw - 1, applied in order (LAPACK's laswp), with
// partial pivoting's p_i >= r0 + i, are one permutation of the rows they touch, and every row's final content has a
// closed form. Row r0 + i is not touched after step i, so it ends with what row p_i held just before step i. A row
// x >= r0 + i holds, before step i, its own content unless an earlier step h moved something into it (p_h = x), and
// then what row r0 + h held before step h. With B(i) = what row r0 + i holds before step i:
//   B(i)       = B(h) for the last h < i with p_h = r0 + i, else row r0 + i's own content;
//   row r0 + i ends with B(h) for the last h < i with p_h = p_i, else row p_i's own content;
//   a row x >= r0 + nsw ends with B(h) for the last h with p_h = x.
// B's links go to smaller indices, so log2(nsw) rounds of pointer jumping find each chain's root. swap_plan builds
// this in shared memory with the CTA's threads: dst[e] / src[e], e < m: after the interchanges row dst[e] holds what
// row src[e] held before them. The first nsw entries are rows r0 .. r0 + nsw in order (some unchanged), then the rows
// below that moved. A pivot out of range (p_i < r0 + i or >= n) is recorded as M25_DEV_INDEX and taken as none.
#define PLAN_MAX 256
static_assert(NB2 <= PLAN_MAX, "an outer panel's interchanges make one plan");
struct SwapPlan {
    int piv[PLAN_MAX];
    int jump[2][PLAN_MAX];
    int low[PLAN_MAX];                 // the source row for a moved row below, else -1
    int dst[2 * PLAN_MAX], src[2 * PLAN_MAX];
    int m;
};

__device__ void swap_plan(const int *ipiv, int r0, int nsw, int n, SwapPlan &P, int *err)
{
    const int T = blockDim.x, t = threadIdx.x;
    for (int i = t; i < nsw; i += T) {
        int p = ipiv[r0 + i];
        if (p < r0 + i || p >= n) {
            dev_error(err, M25_DEV_INDEX);
            p = r0 + i;
        }
        P.piv[i] = p;
    }
    __syncthreads();
    for (int i = t; i < nsw; i += T) {                     // B's link: the last h < i with p_h = r0 + i, else i
        int last = i;
        for (int h = 0; h < i; ++h)
            if (P.piv[h] == r0 + i) last = h;
        P.jump[0][i] = last;
    }
    __syncthreads();
    int cur = 0;
    for (int s = 1; s < nsw; s <<= 1) {
        for (int i = t; i < nsw; i += T) P.jump[cur ^ 1][i] = P.jump[cur][P.jump[cur][i]];
        __syncthreads();
        cur ^= 1;
    }
    for (int i = t; i < nsw; i += T) {
        const int p = P.piv[i];
        int last = -1;
        bool later = false;
        for (int h = 0; h < nsw; ++h)
            if (P.piv[h] == p) {
                if (h < i) last = h;
                else if (h > i) later = true;
            }
        P.dst[i] = r0 + i;
        P.src[i] = last >= 0 ? r0 + P.jump[cur][last] : p;
        P.low[i] = (p >= r0 + nsw && !later) ? r0 + P.jump[cur][i] : -1;
    }
    __syncthreads();
    if (t < 32) {                                          // the moved rows below, in order of i
        int m = nsw;
        for (int b = 0; b < nsw; b += 32) {
            const int i = b + t;
            const bool f = i < nsw && P.low[i] >= 0;
            const unsigned bal = __ballot_sync(0xffffffffu, f);
            if (f) {
                const int e = m + __popc(bal & ((1u << t) - 1u));
                P.dst[e] = P.piv[i];
                P.src[e] = P.low[i];
            }
            m += __popc(bal);
        }
        if (t == 0) P.m = m;
    }
    __syncthreads();
}

// The plan applied to up to COLS columns (cs[j] < 0: none) by a warp, Q entries a lane (P.m <= 32 Q): every source
// of them read before any destination is written (the warp barrier orders the lanes' loads before their stores).
// Entries e < top go to shared memory instead (xs[j * xcol + e * xrow]) when xs is given.
template <typename R, int Q, int COLS>
__device__ __forceinline__ void apply_plan(R *A, long lda, const long (&cs)[COLS], const SwapPlan &P, int lane,
                                           cpx<R> *xs, int top, int xcol, int xrow)
{
    cpx<R> v[COLS][Q];
#pragma unroll
    for (int j = 0; j < COLS; ++j) {
        if (cs[j] < 0) continue;
        const R *col = A + 2 * (size_t)cs[j] * lda;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int e = lane + 32 * q;
            if (e < P.m) v[j][q] = ldc<R>(col, P.src[e]);
        }
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < COLS; ++j) {
        if (cs[j] < 0) continue;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int e = lane + 32 * q;
            if (e < P.m) {
                if (xs && e < top) xs[(size_t)j * xcol + (size_t)e * xrow] = v[j][q];
                else stc<R>(A, (size_t)cs[j] * lda + P.dst[e], v[j][q]);
            }
        }
    }
    __syncwarp();
}

// a warp's columns k .. k + COLS of the two ranges [a0, a1), [b0, b1) (na = a1 - a0, nc in all), the plan applied
template <typename R, int Q, int COLS>
__device__ __forceinline__ void laswp_cols(R *A, long lda, const SwapPlan &P, long a0, long na, long b0, long nc,
                                           int lane, long wid, long nw)
{
    for (long k = wid * COLS; k < nc; k += nw * COLS) {
        long cs[COLS];
#pragma unroll
        for (int j = 0; j < COLS; ++j) {
            const long kk = k + j;
            cs[j] = kk >= nc ? -1 : kk < na ? a0 + kk : b0 + (kk - na);
        }
        apply_plan<R, Q, COLS>(A, lda, cs, P, lane, nullptr, 0, 0, 0);
    }
}

// Interchanges on columns: the plan of rows r0 .. (nsw interchanges) on the columns [a0, a1) and [b0, b1), a warp a
// few columns at a time. blockIdx.y = g > 0 shifts the rows, the interchange count (down) and [a0, a1) by g gs: the
// interchanges of an outer panel's later panels applied to each earlier panel's columns in one launch.
template <typename R>
__global__ void __launch_bounds__(256) k_laswp_plan(R *A, long lda, int n, const int *ipiv, int r0, int nsw, long a0,
                                                    long a1, long b0, long b1, int gs, int *err)
{
    __shared__ SwapPlan P;
    const int g = blockIdx.y;
    r0 += g * gs; nsw -= g * gs; a0 += (long)g * gs; a1 += (long)g * gs;
    swap_plan(ipiv, r0, nsw, n, P, err);
    const long na = a1 - a0, nc = na + (b1 - b0);
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    const long wid = (long)blockIdx.x * wpb + (threadIdx.x >> 5), nw = (long)gridDim.x * wpb;
    if (nsw <= 64) laswp_cols<R, 4, 4>(A, lda, P, a0, na, b0, nc, lane, wid, nw);
    else if (nsw <= 128) laswp_cols<R, 8, 2>(A, lda, P, a0, na, b0, nc, lane, wid, nw);
    else laswp_cols<R, 16, 1>(A, lda, P, a0, na, b0, nc, lane, wid, nw);
}

// A[k0 .. k0 + jb, c0 .. c1) = L11^-1 A[k0 .. k0 + jb, c0 .. c1), L11 = A[k0 .., k0 ..] unit lower (jb <= NB), in
// shared memory; each thread one column
// 64 columns a block of 256 threads: column c = tid % 64, rows split 4 ways (k % 4 == tid / 64); after row i is final
// the block updates the rows below it (one barrier a row)
template <typename R>
__global__ void __launch_bounds__(256) k_trsm(R *A, long lda, int k0, int jb, long c0, long c1)
{
    typedef cpx<R> C;
    extern __shared__ unsigned char sm_raw[];
    C *L = reinterpret_cast<C *>(sm_raw);                  // L[k * NB + i] = L(k, i)
    C *X = L + NB * NB;                                    // X[k * 64 + column]
    for (int e = threadIdx.x; e < jb * jb; e += blockDim.x) {
        int i = e / jb, k = e % jb;                        // column i, row k (coalesced)
        L[k * NB + i] = ldc<R>(A, (size_t)(k0 + i) * lda + k0 + k);
    }
    const int cl = threadIdx.x & 63, g = threadIdx.x >> 6;
    const long c = c0 + blockIdx.x * 64L + cl;
    const bool live = c < c1;
    for (int k = g; k < jb; k += 4) X[k * 64 + cl] = live ? ldc<R>(A, (size_t)c * lda + k0 + k) : mk<R>(0, 0);
    __syncthreads();
    for (int i = 0; i < jb - 1; ++i) {
        const C xi = X[i * 64 + cl];
        for (int k = i + 1 + ((g - (i + 1)) % 4 + 4) % 4; k < jb; k += 4) {
            C x = X[k * 64 + cl];
            cfms<R>(x, L[k * NB + i], xi);
            X[k * 64 + cl] = x;
        }
        __syncthreads();
    }
    if (live)
        for (int k = g; k < jb; k += 4) stc<R>(A, (size_t)c * lda + k0 + k, X[k * 64 + cl]);
}


// The same for a full panel (jb = NB = 64) without a barrier inside the substitution: a warp solves 32
// columns, one a lane, the lane's column in registers (64 complex), L11 in shared memory read as broadcasts. The
// columns are staged through shared memory (a column's stride NB + 1: the lanes' reads of their own columns fall in
// different banks) so that every global load and store is a warp's 256 contiguous bytes. The arithmetic and its
// order are those of k_trsm (row i's multiple subtracted from the rows below, i ascending).
// With SWAP, the panel's own interchanges (ipiv[k0 .. k0 + NB)) are applied to the columns as they are loaded: the
// solved rows come from the plan's sources, and the rows below that move are written back directly (the separate
// interchange launch folded into this one).
template <typename R, int T64_WARPS, bool SWAP>
__global__ void __launch_bounds__(32 * T64_WARPS) k_trsm64(R *A, long lda, int k0, long c0, long c1, const int *ipiv,
                                                           int n, int *err)
{
    typedef cpx<R> C;
    typedef typename vec2_of<R>::type V;
    constexpr int XS = NB + 1;
    extern __shared__ __align__(16) unsigned char t64_raw[];
    __shared__ SwapPlan P;
    C *L = reinterpret_cast<C *>(t64_raw);                   // L[i * NB + k] = L11(k, i)
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    C *Xs = L + NB * NB + (size_t)w * 32 * XS;
    const V *A2 = reinterpret_cast<const V *>(A);
    static_assert(NB * NB % (8 * 32 * T64_WARPS) == 0, "L11 in whole batches");
    if (SWAP) swap_plan(ipiv, k0, NB, n, P, err);
    for (int e0 = threadIdx.x; e0 < NB * NB; e0 += 8 * 32 * T64_WARPS) {     // 8 loads in flight a thread
        V v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int e = e0 + q * 32 * T64_WARPS, i = e / NB, k = e % NB;
            v[q] = A2[(size_t)(k0 + i) * lda + k0 + k];
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) L[e0 + q * 32 * T64_WARPS] = mk<R>(v[q].x, v[q].y);
    }
    const long cbase = c0 + ((long)blockIdx.x * T64_WARPS + w) * 32;
    if (SWAP) {                                             // 4 rows x 8 (4) columns of loads in flight a lane
        constexpr int SC = sizeof(R) == 4 ? 8 : 4;
        for (int c8 = 0; c8 < 32; c8 += SC) {
            long cs[SC];
#pragma unroll
            for (int j = 0; j < SC; ++j) cs[j] = cbase + c8 + j < c1 ? cbase + c8 + j : -1;
            apply_plan<R, 4, SC>(A, lda, cs, P, lane, Xs + c8 * XS, NB, XS, 1);
        }
    } else for (int c8 = 0; c8 < 32; c8 += 8) {             // 16 loads in flight a lane
        V v[8][2];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const long c = cbase + c8 + q;
            if (c < c1) {
                const V *src = A2 + (size_t)c * lda + k0;
                v[q][0] = src[lane];
                v[q][1] = src[lane + 32];
            }
        }
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (cbase + c8 + q < c1) {
                Xs[(c8 + q) * XS + lane] = mk<R>(v[q][0].x, v[q][0].y);
                Xs[(c8 + q) * XS + lane + 32] = mk<R>(v[q][1].x, v[q][1].y);
            }
    }
    __syncthreads();
    // by blocks of 16 rows (the unrolled code of two 16 x 16 steps stays in the instruction cache): the diagonal
    // block solved in registers, then its multiples subtracted from each block below; every entry still takes its
    // terms in ascending i
    C *xs = Xs + lane * XS;
    for (int d = 0; d < NB / 16; ++d) {
        C xd[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) xd[k] = xs[d * 16 + k];
#pragma unroll
        for (int i = 0; i < 15; ++i) {
#pragma unroll
            for (int k = i + 1; k < 16; ++k) cfms<R>(xd[k], L[(d * 16 + i) * NB + d * 16 + k], xd[i]);
        }
#pragma unroll
        for (int k = 0; k < 16; ++k) xs[d * 16 + k] = xd[k];
        for (int e = d + 1; e < NB / 16; ++e) {
            C xe[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) xe[k] = xs[e * 16 + k];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
#pragma unroll
                for (int k = 0; k < 16; ++k) cfms<R>(xe[k], L[(d * 16 + i) * NB + e * 16 + k], xd[i]);
            }
#pragma unroll
            for (int k = 0; k < 16; ++k) xs[e * 16 + k] = xe[k];
        }
    }
    __syncwarp();
    V *D2 = reinterpret_cast<V *>(A);
    for (int cc = 0; cc < 32; ++cc) {
        const long c = cbase + cc;
        if (c < c1) {
            V *dst = D2 + (size_t)c * lda + k0;
            const C v0 = Xs[cc * XS + lane], v1 = Xs[cc * XS + lane + 32];
            V w0, w1;
            w0.x = v0.x; w0.y = v0.y; w1.x = v1.x; w1.y = v1.y;
            dst[lane] = w0;
            dst[lane + 32] = w1;
        }
    }
}
template <typename R> constexpr int t64_warps() { return sizeof(R) == 4 ? 4 : 2; }
template <typename R> constexpr size_t t64_smem()
{
    return sizeof(cpx<R>) * (NB * NB + (size_t)t64_warps<R>() * 32 * (NB + 1));
}

// U12 of a whole outer panel in one launch: rows [K0, K0 + JB) (JB <= NB2) of the columns [c0, c1), after the outer
// panel's interchanges (ipiv[K0 .. K0 + JB), applied as a plan; the rows below that move written back directly),
// U12 = L11^-1 A12 with L11 = A[K0 .., K0 ..] unit lower. TO_COLS columns a CTA of 256 threads (a warp a column),
// their JB rows in shared memory. By 64-row blocks: the diagonal block of L11 staged in shared memory, each warp
// solves its column's 64 rows (two rows a lane in registers, the solved value passed by shuffle), then every thread
// takes a row below the block and subtracts the block's multiples from it for all the CTA's columns (L read from
// the factor, coalesced across the threads). Each entry takes its terms x -= L(k, i) x_i in ascending i, as a
// forward substitution does; FP32 (FP64) on the CUDA cores throughout.
#define TO_COLS 8
#define TO_THREADS 256
static_assert(TO_COLS * 32 == TO_THREADS, "a warp a column");
template <typename R> constexpr size_t to_smem() { return sizeof(cpx<R>) * ((size_t)NB2 * TO_COLS + NB * (NB + 1)); }

template <typename R>
__global__ void __launch_bounds__(TO_THREADS) k_trsm_outer(R *A, long lda, int n, int K0, int JB, const int *ipiv,
                                                           long c0, long c1, int *err)
{
    typedef cpx<R> C;
    extern __shared__ __align__(16) unsigned char to_raw[];
    __shared__ SwapPlan P;
    C *X = reinterpret_cast<C *>(to_raw);                 // X[r * TO_COLS + j]: row K0 + r of the CTA's column j
    C *Lb = X + (size_t)NB2 * TO_COLS;                     // Lb[i * (NB + 1) + k] = L11(kb + k, kb + i)
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const long cw = c0 + (long)blockIdx.x * TO_COLS + w;    // this warp's column
    swap_plan(ipiv, K0, JB, n, P, err);
    {
        long cs[1] = {cw < c1 ? cw : -1};
        apply_plan<R, 2 * PLAN_MAX / 32, 1>(A, lda, cs, P, lane, X + w, JB, 0, TO_COLS);
        if (cw >= c1)
            for (int r = lane; r < JB; r += 32) X[r * TO_COLS + w] = mk<R>(0, 0);
    }
    for (int kb = 0; kb < JB; kb += NB) {
        const int jb = min(NB, JB - kb);
        __syncthreads();                                   // (X complete; the previous block's Lb reads done)
        for (int e = t; e < jb * jb; e += TO_THREADS) {
            const int i = e / jb, k = e % jb;
            Lb[i * (NB + 1) + k] = ldc<R>(A, (size_t)(K0 + kb + i) * lda + K0 + kb + k);
        }
        __syncthreads();
        {                                                  // the diagonal block, warp w's column
            C x0 = lane < jb ? X[(kb + lane) * TO_COLS + w] : mk<R>(0, 0);
            C x1 = lane + 32 < jb ? X[(kb + lane + 32) * TO_COLS + w] : mk<R>(0, 0);
            for (int i = 0; i < jb - 1; ++i) {
                const C s = i < 32 ? x0 : x1;
                C xi;
                xi.x = __shfl_sync(0xffffffffu, s.x, i & 31);
                xi.y = __shfl_sync(0xffffffffu, s.y, i & 31);
                if (lane > i && lane < jb) cfms<R>(x0, Lb[i * (NB + 1) + lane], xi);
                if (lane + 32 > i && lane + 32 < jb) cfms<R>(x1, Lb[i * (NB + 1) + lane + 32], xi);
            }
            if (lane < jb) X[(kb + lane) * TO_COLS + w] = x0;
            if (lane + 32 < jb) X[(kb + lane + 32) * TO_COLS + w] = x1;
        }
        __syncthreads();
        for (int r = kb + jb + t; r < JB; r += TO_THREADS) {   // the rows below the block
            C x[TO_COLS];
#pragma unroll
            for (int j = 0; j < TO_COLS; ++j) x[j] = X[r * TO_COLS + j];
            const R *lr = A + 2 * ((size_t)(K0 + kb) * lda + K0 + r);
#pragma unroll 8
            for (int i = 0; i < jb; ++i) {
                const C l = ldc<R>(lr, (size_t)i * lda);
#pragma unroll
                for (int j = 0; j < TO_COLS; ++j) cfms<R>(x[j], l, X[(kb + i) * TO_COLS + j]);
            }
#pragma unroll
            for (int j = 0; j < TO_COLS; ++j) X[r * TO_COLS + j] = x[j];
        }
    }
    __syncthreads();
    if (cw < c1)
        for (int r = lane; r < JB; r += 32) stc<R>(A, (size_t)cw * lda + K0 + r, X[r * TO_COLS + w]);
}

// C (M x N) -= A (M x K) B (K x N), all column-major complex inside the factor (lda). A 128 x 64 tile per block of
// 256 threads, each 8 x 4 outputs; K staged BK at a time through two shared-memory buffers, the next slice loaded
// into registers while the current one is multiplied (one barrier a slice).
template <typename R>
__global__ void __launch_bounds__(256) k_gemm_update(R *Cm, const R *Am, const R *Bm, long lda, int M, int N, int K)
{
    typedef cpx<R> C;
    constexpr int BM = 128, BN = 64, BK = 8;
    extern __shared__ unsigned char gemm_raw[];
    C(*As)[BK][BM] = reinterpret_cast<C(*)[BK][BM]>(gemm_raw);                       // [2][BK][BM]
    C(*Bs)[BK][BN + 1] = reinterpret_cast<C(*)[BK][BN + 1]>(gemm_raw + 2 * sizeof(C) * BK * BM);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    C acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = mk<R>(0, 0);
    // each thread stages 4 A and 2 B elements a slice
    C ra[4], rb[2];
    auto load = [&](int kk) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            int e = threadIdx.x + 256 * u, k = e / BM, m = e % BM;
            ra[u] = (m0 + m < M && kk + k < K) ? ldc<R>(Am, (size_t)(kk + k) * lda + m0 + m) : mk<R>(0, 0);
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            int e = threadIdx.x + 256 * u, nn = e / BK, k = e % BK;
            rb[u] = (n0 + nn < N && kk + k < K) ? ldc<R>(Bm, (size_t)(n0 + nn) * lda + kk + k) : mk<R>(0, 0);
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int u = 0; u < 4; ++u) { int e = threadIdx.x + 256 * u; As[buf][e / BM][e % BM] = ra[u]; }
#pragma unroll
        for (int u = 0; u < 2; ++u) { int e = threadIdx.x + 256 * u; Bs[buf][e % BK][e / BK] = rb[u]; }
    };
    load(0);
    store(0);
    __syncthreads();
    int buf = 0;
    for (int kk = 0; kk < K; kk += BK) {
        const bool more = kk + BK < K;
        if (more) load(kk + BK);
#pragma unroll
        for (int k = 0; k < BK; ++k) {
            C a[8], b[4];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = As[buf][k][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[buf][k][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) cfma<R>(acc[i][j], a[i], b[j]);
        }
        if (more) store(buf ^ 1);
        __syncthreads();
        buf ^= 1;
    }
    // C -= the product, four rows of outputs at a time: their 16 values of C read before any is written (a load ->
    // store chain a value serialised the memory latency 32 times a thread)
#pragma unroll
    for (int i0 = 0; i0 < 8; i0 += 4) {
        C cv[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int m = m0 + ty + 16 * (i0 + i), nn = n0 + tx + 16 * j;
                cv[i][j] = (m < M && nn < N) ? ldc<R>(Cm, (size_t)nn * lda + m) : mk<R>(0, 0);
            }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int m = m0 + ty + 16 * (i0 + i), nn = n0 + tx + 16 * j;
                if (m < M && nn < N) stc<R>(Cm, (size_t)nn * lda + m, cv[i][j] - acc[i0 + i][j]);
            }
    }
}

// The complex128 update C -= A B on the FP64 tensor cores (mma.sync m8n8k4 f64; Blackwell's tcgen05 has no FP64
// kind). Column-major A (M x K), B (K x N), C (M x N), one leading dimension. A 64 x 64 tile a CTA of four warps,
// each warp 32 x 32 complex: 2 x 4 tiles of 16 x 8 (mma m16n8k8) for the real and the imaginary part,
// C_re -= A_re B_re - A_im B_im, C_im -= A_re B_im + A_im B_re (four real products). K in slices of 16 copied into
// shared memory by cp.async (double-buffered), one 16-byte copy and one 16-byte fragment read a complex number.
#define ZD_BM 64
#define ZD_BN 64
#define ZD_BK 16
#define ZD_SA (ZD_BM + 2)          // A slice [k][m], complex: a row stride = 2 mod 8 keeps the 16-byte reads conflict-free
#define ZD_SB (ZD_BK + 4)          // B slice [n][k], complex: 4 mod 8


__device__ __forceinline__ void cp_async16_zfill_lu(void *smem, const void *gmem, bool valid)
{
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(sa), "l"(gmem), "r"(valid ? 16 : 0) : "memory");
}

static size_t zdmma_smem() { return sizeof(double2) * 2 * ((size_t)ZD_BK * ZD_SA + (size_t)ZD_BN * ZD_SB); }

__global__ void __launch_bounds__(128, 2) k_zgemm_dmma(double *Cm, const double *Am, const double *Bm, long lda, int M,
                                                       int N, int K)
{
    extern __shared__ __align__(16) double2 zd_raw[];
    typedef double2 ASlice[ZD_BK][ZD_SA];
    typedef double2 BSlice[ZD_BN][ZD_SB];
    ASlice *As = reinterpret_cast<ASlice *>(zd_raw);                           // [buf]
    BSlice *Bs = reinterpret_cast<BSlice *>(zd_raw + 2 * ZD_BK * ZD_SA);       // [buf]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m0 = blockIdx.y * ZD_BM, n0 = blockIdx.x * ZD_BN;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
    double cr[2][4][4], ci[2][4][4];                 // [16-row tile][8-column tile][fragment]
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 4; ++q) cr[i][j][q] = ci[i][j][q] = 0.0;
    const double2 *A2 = reinterpret_cast<const double2 *>(Am), *B2 = reinterpret_cast<const double2 *>(Bm);
    // a K slice into buffer buf: one 16-byte asynchronous copy a complex number
    auto stage = [&](int buf, int kk) {
        for (int e = tid; e < ZD_BM * ZD_BK; e += 128) {
            const int k = e / ZD_BM, m = e % ZD_BM;                               // A: m fastest (contiguous)
            const bool ok = m0 + m < M && kk + k < K;
            cp_async16_zfill_lu(&As[buf][k][m], A2 + (ok ? (size_t)(kk + k) * lda + m0 + m : 0), ok);
        }
        for (int e = tid; e < ZD_BN * ZD_BK; e += 128) {
            const int nn = e / ZD_BK, k = e % ZD_BK;                              // B: k fastest (contiguous)
            const bool ok = n0 + nn < N && kk + k < K;
            cp_async16_zfill_lu(&Bs[buf][nn][k], B2 + (ok ? (size_t)(n0 + nn) * lda + kk + k : 0), ok);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    stage(0, 0);
    int buf = 0;
    const int fg = lane >> 2, ft = lane & 3;       // fragment coordinates (group, thread in group)
    for (int kk = 0; kk < K; kk += ZD_BK) {
        if (kk + ZD_BK < K) stage(buf ^ 1, kk + ZD_BK);                           // the next slice, other buffer
        else asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 1;" ::: "memory");
        __syncthreads();
#pragma unroll
        for (int k8 = 0; k8 < ZD_BK; k8 += 8) {
            double ar[2][4], ai[2][4], nai[2][4], br[4][2], bi[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int r = wm + 16 * i + fg;
                const double2 v0 = As[buf][k8 + ft][r], v1 = As[buf][k8 + ft][r + 8];
                const double2 v2 = As[buf][k8 + ft + 4][r], v3 = As[buf][k8 + ft + 4][r + 8];
                ar[i][0] = v0.x; ai[i][0] = v0.y;
                ar[i][1] = v1.x; ai[i][1] = v1.y;
                ar[i][2] = v2.x; ai[i][2] = v2.y;
                ar[i][3] = v3.x; ai[i][3] = v3.y;
#pragma unroll
                for (int q = 0; q < 4; ++q) nai[i][q] = -ai[i][q];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = wn + 8 * j + fg;
                const double2 w0 = Bs[buf][c][k8 + ft], w1 = Bs[buf][c][k8 + ft + 4];
                br[j][0] = w0.x; bi[j][0] = w0.y;
                br[j][1] = w1.x; bi[j][1] = w1.y;
            }
            // two passes over the 8 tiles: independent products between two into the same accumulator
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    dmma_16x8x8(cr[i][j], ar[i], br[j]);
                    dmma_16x8x8(ci[i][j], ar[i], bi[j]);
                }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    dmma_16x8x8(cr[i][j], nai[i], bi[j]);
                    dmma_16x8x8(ci[i][j], ai[i], br[j]);
                }
        }
        __syncthreads();                                                          // the buffer is the next stage's
        buf ^= 1;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    // C -= the product: fragment q of tile (i, j) is row g (+ 8 for q >= 2), column 2 t + (q & 1). By 16-row tile,
    // its 16 values of C read before any is written (a load -> store chain a value serialised the memory latency
    // 32 times a thread; the complex128 LU at N = 18,788 took 705 ms with it, 626 ms without)
    double2 *C2 = reinterpret_cast<double2 *>(Cm);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        double2 cv[4][4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int m = m0 + wm + 16 * i + fg + (q >= 2 ? 8 : 0), nn = n0 + wn + 8 * j + 2 * ft + (q & 1);
                cv[q][j] = (m < M && nn < N) ? C2[(size_t)nn * lda + m] : make_double2(0.0, 0.0);
            }
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int m = m0 + wm + 16 * i + fg + (q >= 2 ? 8 : 0), nn = n0 + wn + 8 * j + 2 * ft + (q & 1);
                if (m < M && nn < N) C2[(size_t)nn * lda + m] = make_double2(cv[q][j].x - cr[i][j][q],
                                                                             cv[q][j].y - ci[i][j][q]);
            }
    }
}

template <typename R>
static size_t gemm_smem() { return 2 * sizeof(cpx<R>) * 8 * 128 + 2 * sizeof(cpx<R>) * 8 * 65; }

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

// ---- solves with diagonal-block inverses (the reference's GPU solve design, gpu_vk.py:242-290) -----------------------
// Once per factorisation (k_block_inverses): for every diagonal block of TB rows, inv(L_bb) (unit lower) and
// inv(U_bb) (upper), one CTA a block, thread j forming column j of each. Per solve (k_trsv_step): one launch per
// block; every CTA applies the block's inverse (transposed) to the block's running right-hand sides, CTA 0 stores
// the result, and all CTAs update the right-hand sides of the unknowns still to come (a contiguous factor segment
// per unknown, a warp per unknown).
template <typename R>
__global__ void __launch_bounds__(TB) k_block_inverses(const R *A, long lda, int n, R *inv)
{
    typedef cpx<R> C;
    extern __shared__ unsigned char inv_raw[];
    C(*D)[TB + 1] = reinterpret_cast<C(*)[TB + 1]>(inv_raw);          // D[r][c] = A[b0 + r, b0 + c]
    C(*X)[TB + 1] = reinterpret_cast<C(*)[TB + 1]>(inv_raw + sizeof(C) * TB * (TB + 1));   // column j: thread j
    const int b = blockIdx.x, b0 = b * TB, bs = min(TB, n - b0), j = threadIdx.x;
    for (int e = threadIdx.x; e < TB * TB; e += blockDim.x) {
        int c = e / TB, r = e % TB;                         // identity outside the block's bs x bs corner
        D[r][c] = (r < bs && c < bs) ? ldc<R>(A, (size_t)(b0 + c) * lda + b0 + r) : mk<R>(r == c ? 1 : 0, 0);
    }
    __syncthreads();
    R *iL = inv + 2 * ((size_t)b * 2 * TB * TB), *iU = iL + 2 * (size_t)TB * TB;     // [r][c] row-major
    // column j of inv(L), L unit lower: x_i = delta_ij - sum_{j <= k < i} L[i][k] x_k
    for (int i = 0; i < TB; ++i) {
        C v = mk<R>(i == j ? 1 : 0, 0);
        for (int k = j; k < i; ++k) cfms<R>(v, D[i][k], X[k][j]);
        X[i][j] = i < j ? mk<R>(0, 0) : v;
    }
    for (int i = 0; i < TB; ++i) stc<R>(iL, (size_t)i * TB + j, X[i][j]);
    // column j of inv(U): x_j = 1 / U[j][j]; x_i = -(sum_{i < k <= j} U[i][k] x_k) / U[i][i], i = j-1 .. 0
    for (int i = TB - 1; i >= 0; --i) {
        C v = mk<R>(0, 0);
        if (i == j) v = cdiv<R>(mk<R>(1, 0), D[j][j]);
        else if (i < j) {
            for (int k = i + 1; k <= j; ++k) cfma<R>(v, D[i][k], X[k][j]);
            v = cdiv<R>(mk<R>(-v.x, -v.y), D[i][i]);
        }
        X[i][j] = v;
    }
    for (int i = 0; i < TB; ++i) stc<R>(iU, (size_t)i * TB + j, X[i][j]);
}

// The whole triangular solve in one cooperative launch, no kernel boundary between blocks. CTA g owns the row blocks
// [bb0, bb1) (contiguous) and keeps their running right-hand sides in shared memory. Blocks are visited in solve
// order (forward: 0 .. nb-1 for U^T; backward: nb-1 .. 0 for L^T):
//   a block of another CTA that precedes mine: wait for its flag (bounded), read its solved values, apply them to
//     my rows (the factor's column segment of each of my rows: contiguous);
//   a block of mine: every earlier block has been applied to it, so solve it with its inverse (transposed),
//     publish the values (store, fence, flag = epoch), then apply them to my other rows still to come.
// The flags only point backwards in solve order and all CTAs are co-resident: no cycle, every wait ends.
template <typename R>
struct TrsvArgs {
    const R *A; long lda; int n; int nb;
    const R *inv;          // block inverses: per block, inv(L_bb) then inv(U_bb), TB x TB row-major each
    const R *Tin;          // right-hand sides (n x nrhs)
    R *Xout;               // solution (n x nrhs)
    int nrhs; int backward;
    int *flags; const int *epoch_ptr; int *err;   // flags[b] == *epoch_ptr: block b solved in this call
};

__global__ void k_bump_epoch(int *e) { *e += 1; }

template <typename R>
__global__ void __launch_bounds__(256) k_trsv_persistent(TrsvArgs<R> a)
{
    typedef cpx<R> C;
    extern __shared__ unsigned char tp_raw[];
    const int G = gridDim.x, g = blockIdx.x, nb = a.nb, nrhs = a.nrhs;
    const int epoch = *(volatile const int *)a.epoch_ptr;
    const int per = (nb + G - 1) / G, bb0 = g * per, bb1 = min(nb, bb0 + per);
    const int R0 = bb0 * TB, R1 = min(a.n, bb1 * TB), nr = max(0, R1 - R0);
    C(*Ws)[TB + 1] = reinterpret_cast<C(*)[TB + 1]>(tp_raw);
    C(*Yb)[16] = reinterpret_cast<C(*)[16]>(tp_raw + sizeof(C) * TB * (TB + 1));
    C(*T)[16] = reinterpret_cast<C(*)[16]>(tp_raw + sizeof(C) * (TB * (TB + 1) + TB * 16));
    __shared__ int ok;
    for (int e = threadIdx.x; e < nr * nrhs; e += blockDim.x)
        T[e / nrhs][e % nrhs] = ldc<R>(a.Tin, (size_t)(R0 + e / nrhs) * nrhs + e % nrhs);
    if (threadIdx.x == 0) ok = 1;
    __syncthreads();
    if (nr == 0) return;
    // one lane a row: lane l of warp w takes row ra + 32 w + l (+ 256 per round) and streams its factor segment
    // A[b0 .. b0 + bs, r] (contiguous) against Yb (a shared-memory broadcast); no reductions across lanes
    auto prefetch = [&](int b0, int bs, int ra, int rb) {          // the segments into L1 while the flag is awaited
        for (int r = ra + threadIdx.x; r < rb; r += blockDim.x) {
            const char *p = reinterpret_cast<const char *>(a.A + 2 * ((size_t)r * a.lda + b0));
            for (int off = 0; off < bs * (int)sizeof(C); off += 128) asm volatile("prefetch.global.L1 [%0];" ::"l"(p + off));
        }
    };
    auto apply = [&](int b0, int bs, int ra, int rb, bool) {
        for (int r = ra + threadIdx.x; r < rb; r += blockDim.x) {
            const C *seg = reinterpret_cast<const C *>(a.A) + (size_t)r * a.lda + b0;
            C acc[16];
#pragma unroll
            for (int c = 0; c < 16; ++c) acc[c] = mk<R>(0, 0);
#pragma unroll 4
            for (int k = 0; k < bs; ++k) {
                const C v = seg[k];
#pragma unroll
                for (int c = 0; c < 16; ++c)
                    if (c < nrhs) cfma<R>(acc[c], v, Yb[k][c]);
            }
#pragma unroll
            for (int c = 0; c < 16; ++c)
                if (c < nrhs) T[r - R0][c] -= acc[c];
        }
    };
    bool ws_ready = false;
    {                                                               // my first block's inverse, ahead of time
        const int first = a.backward ? bb1 - 1 : bb0;
        const int fs = min(TB, a.n - first * TB);
        const R *W = a.inv + 2 * ((size_t)first * 2 * TB * TB + (a.backward ? 0 : (size_t)TB * TB));
        for (int e = threadIdx.x; e < fs * TB; e += blockDim.x) Ws[e / TB][e % TB] = ldc<R>(W, e);
        ws_ready = true;
        __syncthreads();
    }
    for (int step = 0; step < nb; ++step) {
        const int b = a.backward ? nb - 1 - step : step;
        const int b0 = b * TB, bs = min(TB, a.n - b0);
        const bool mine = b >= bb0 && b < bb1;
        const bool before_mine = a.backward ? b >= bb1 : b < bb0;
        if (!mine && !before_mine) break;                           // blocks after mine do not touch my rows
        if (!mine) {
            prefetch(b0, bs, R0, R1);                               // the factor reads do not wait for the flag
            if (threadIdx.x == 0) {
                long it = 0;
                while (ld_acquire_u32((const unsigned *)(a.flags + b)) != (unsigned)epoch) {
                    if (++it > (1L << 26) || *(volatile int *)a.err) { ok = 0; dev_error(a.err, M25_DEV_TIMEOUT); break; }
                    __nanosleep(32);
                }
            }
            __syncthreads();
            if (!ok) return;
            for (int e = threadIdx.x; e < bs * nrhs; e += blockDim.x) {       // another CTA's values: past L1
                const R *p = a.Xout + 2 * ((size_t)(b0 + e / nrhs) * nrhs + e % nrhs);
                Yb[e / nrhs][e % nrhs] = mk<R>(__ldcg(p), __ldcg(p + 1));
            }
            __syncthreads();
            apply(b0, bs, R0, R1, true);                            // every row of mine comes after it
            __syncthreads();
            continue;
        }
        // my block: solve it (its inverse staged at the start or after my previous block), publish, apply to my
        // remaining rows
        if (!ws_ready) {
            const R *W = a.inv + 2 * ((size_t)b * 2 * TB * TB + (a.backward ? 0 : (size_t)TB * TB));
            for (int e = threadIdx.x; e < bs * TB; e += blockDim.x) Ws[e / TB][e % TB] = ldc<R>(W, e);
        }
        ws_ready = false;
        __syncthreads();
        for (int e = threadIdx.x; e < bs * nrhs; e += blockDim.x) {
            int rr = e / nrhs, c = e % nrhs;
            C acc = mk<R>(0, 0);
            for (int k = 0; k < bs; ++k) cfma<R>(acc, Ws[k][rr], T[b0 - R0 + k][c]);
            Yb[rr][c] = acc;
        }
        __syncthreads();
        for (int e = threadIdx.x; e < bs * nrhs; e += blockDim.x)
            stc<R>(a.Xout, (size_t)(b0 + e / nrhs) * nrhs + e % nrhs, Yb[e / nrhs][e % nrhs]);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) atomicExch(a.flags + b, epoch);
        // the next own block's inverse, while the rows are updated (Ws is free: this block's y is in Yb)
        const int nxt = a.backward ? b - 1 : b + 1;
        if (nxt >= bb0 && nxt < bb1) {
            const int ns = min(TB, a.n - nxt * TB);
            const R *W = a.inv + 2 * ((size_t)nxt * 2 * TB * TB + (a.backward ? 0 : (size_t)TB * TB));
            for (int e = threadIdx.x; e < ns * TB; e += blockDim.x) Ws[e / TB][e % TB] = ldc<R>(W, e);
            ws_ready = true;
        }
        if (a.backward) apply(b0, bs, R0, b0, false);               // my earlier rows
        else apply(b0, bs, b0 + bs, R1, false);                     // my later rows
        __syncthreads();
    }
}

// The complex64 triangular solve with the factor streamed through shared memory. Same ownership, flags and order
// as k_trsv_persistent; what changes is how the work between two flags is done:
//   - the factor tile of my rows x a block's columns is copied into shared memory by cp.async one task ahead (the
//     copy of the next block's tile runs while this one waits for its flag and computes);
//   - the apply T[r] -= A[r, b] y_b and the block solve y_b = W_b t_b are one shared-memory product (tile_mul):
//     TPR threads a row split the columns (k mod TPR), the KR right-hand sides a compile-time count (the padding
//     columns stay zero), y read as 16-byte pairs;
//   - the inverses of my blocks are staged transposed, both at the start where a CTA owns two blocks;
//   - a block is published by one fence of one thread after the CTA's barrier.
// A task is (block, up to TRSV_RT rows); a CTA owns at most TRSV_MAXPER blocks.
#define TRSV_RT 128
#define TRSV_TBP (TB + 2)          // tile / inverse row stride in elements: 528 bytes, a multiple of 16
#define TRSV_YS 18                 // y row stride: 144 bytes (16-byte aligned rows)
#define TRSV_TS 18                 // running right-hand sides' row stride (144 bytes: conflict-free 16-byte reads)
#define TRSV_MAXPER 5
#define TRSV_NT 256

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// complex64: 128-row tiles and both inverses where a CTA owns two blocks; complex128 (16-byte entries): 32-row
// tiles and one inverse buffer, so that a CTA of two blocks stays within shared memory
template <typename R> constexpr int trsv_rt() { return sizeof(R) == 4 ? TRSV_RT : TRSV_RT / 4; }
template <typename R> constexpr int trsv_nwmax() { return sizeof(R) == 4 ? 2 : 1; }
template <typename R>
static size_t trsv_pipe_smem(int per)
{
    typedef cpx<R> C;
    const int nw = per <= trsv_nwmax<R>() ? per : 1;
    return sizeof(C) * (2 * (size_t)trsv_rt<R>() * TRSV_TBP + (size_t)nw * TB * TRSV_TBP + TB * TRSV_YS +
                        (size_t)per * TB * TRSV_TS);
}

// out[r][c] (-)= sum_{k < kdim} M[r][k] X[k][c] for r < nrows (<= NT / TPR), c < KR; M rows of stride TRSV_TBP,
// X rows of stride xs (16-byte aligned), out rows of stride os. All threads of the CTA call it.
template <int KR, int TPR, bool SUB, typename R>
__device__ __forceinline__ void tile_mul(const cpx<R> *M, int nrows, int kdim, const cpx<R> *X, int xs, cpx<R> *out,
                                         int os)
{
    typedef cpx<R> C;
    const int r = threadIdx.x / TPR, h = threadIdx.x % TPR;
    C acc[KR];
#pragma unroll
    for (int c = 0; c < KR; ++c) acc[c] = mk<R>(0, 0);
    auto term = [&](const C *row, int k) {
        const C v = row[k];
        if constexpr (sizeof(R) == 4) {                      // y as 16-byte pairs
            const float4 *x = reinterpret_cast<const float4 *>(X + (size_t)k * xs);
#pragma unroll
            for (int c2 = 0; c2 < (KR + 1) / 2; ++c2) {
                const float4 y = x[c2];
                cfma<float>(acc[2 * c2], v, mk<float>(y.x, y.y));
                if (2 * c2 + 1 < KR) cfma<float>(acc[2 * c2 + 1], v, mk<float>(y.z, y.w));
            }
        } else {                                             // one 16-byte entry
            const double2 *x = reinterpret_cast<const double2 *>(X + (size_t)k * xs);
#pragma unroll
            for (int c = 0; c < KR; ++c) {
                const double2 y = x[c];
                cfma<double>(acc[c], v, mk<double>(y.x, y.y));
            }
        }
    };
    if (r < nrows) {
        const C *row = M + (size_t)r * TRSV_TBP;
        bool whole = false;
        if constexpr (sizeof(R) == 4) {
            if (kdim == TB) {
                // complex64, a whole block: a compile-time trip count, by batches of U terms whose shared-memory
                // reads all come before their products (N = 18,788, 8 columns: 2.92-2.98 ms a pair against 3.37
                // unbatched, about 3.0 with batches of 2 or 4; the same for complex128, two terms a batch, took
                // 10.6 against 10.1 ms)
                constexpr int U = 8, NY = (KR + 1) / 2;
                static_assert((TB / TPR) % U == 0, "whole batches of a thread's terms");
#pragma unroll
                for (int i0 = 0; i0 < TB / TPR; i0 += U) {
                    C v[U];
                    float4 y[U][NY];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int k = h + TPR * (i0 + u);
                        v[u] = row[k];
                        const float4 *x = reinterpret_cast<const float4 *>(X + (size_t)k * xs);
#pragma unroll
                        for (int q = 0; q < NY; ++q) y[u][q] = x[q];
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u)
#pragma unroll
                        for (int q = 0; q < NY; ++q) {
                            cfma<float>(acc[2 * q], v[u], mk<float>(y[u][q].x, y[u][q].y));
                            if (2 * q + 1 < KR) cfma<float>(acc[2 * q + 1], v[u], mk<float>(y[u][q].z, y[u][q].w));
                        }
                }
                whole = true;
            }
        }
        if (!whole) {
#pragma unroll 2
            for (int k = h; k < kdim; k += TPR) term(row, k);
        }
    }
#pragma unroll
    for (int c = 0; c < KR; ++c)
#pragma unroll
        for (int o = 1; o < TPR; o <<= 1) {
            acc[c].x += __shfl_xor_sync(0xffffffffu, acc[c].x, o);
            acc[c].y += __shfl_xor_sync(0xffffffffu, acc[c].y, o);
        }
    if (r < nrows && h == 0) {
#pragma unroll
        for (int c = 0; c < KR; ++c) {
            if (SUB) out[(size_t)r * os + c] -= acc[c];
            else out[(size_t)r * os + c] = acc[c];
        }
    }
}

template <typename R, int KR>
__global__ void __launch_bounds__(TRSV_NT) k_trsv_pipe(TrsvArgs<R> a, int vec16)
{
    typedef cpx<R> C;
    constexpr int RT = trsv_rt<R>();
    extern __shared__ __align__(16) unsigned char tq_raw[];
    const int G = gridDim.x, g = blockIdx.x, nb = a.nb, nrhs = a.nrhs, n = a.n;
    const int epoch = *(volatile const int *)a.epoch_ptr;
    const int per = (nb + G - 1) / G, bb0 = g * per, bb1 = min(nb, bb0 + per);
    const int R0 = bb0 * TB, R1 = min(n, bb1 * TB), nr = max(0, R1 - R0);
    const int nw = per <= trsv_nwmax<R>() ? per : 1;                        // inverse buffers
    C *tile = reinterpret_cast<C *>(tq_raw);                                // [2][RT][TRSV_TBP]
    C *Wt = tile + 2 * RT * TRSV_TBP;                                       // [nw][TB][TRSV_TBP], transposed
    C *Yb = Wt + (size_t)nw * TB * TRSV_TBP;                                // [TB][TRSV_YS]
    C *T = Yb + TB * TRSV_YS;                                               // [per * TB][TRSV_TS]
    __shared__ int ok;
    if (nr == 0) return;
    for (int e = threadIdx.x; e < nr * TRSV_TS; e += blockDim.x) {
        const int r = e / TRSV_TS, c = e % TRSV_TS;
        T[e] = c < nrhs ? ldc<R>(a.Tin, (size_t)(R0 + r) * nrhs + c) : mk<R>(0, 0);
    }
    for (int e = threadIdx.x; e < TB * TRSV_YS; e += blockDim.x) Yb[e] = mk<R>(0, 0);
    if (threadIdx.x == 0) ok = 1;
    const C *Ac = reinterpret_cast<const C *>(a.A);
    auto blk = [&](int st) { return a.backward ? nb - 1 - st : st; };
    const int s_last = a.backward ? nb - 1 - bb0 : bb1 - 1;
    auto rows_of = [&](int b, int &ra, int &rb) {
        if (b >= bb0 && b < bb1) {
            const int b0 = b * TB, bs = min(TB, n - b0);
            if (a.backward) { ra = R0; rb = b0; } else { ra = b0 + bs; rb = R1; }
        } else { ra = R0; rb = R1; }
    };
    // ---- the tile copies, one task ahead --------------------------------------------------------------------------
    int ls = 0, lc = 0, issued = 0;
    auto issue_next = [&]() {
        int ra = 0, rb = 0;
        while (ls <= s_last) {
            rows_of(blk(ls), ra, rb);
            const int nch = rb > ra ? (rb - ra + RT - 1) / RT : 0;
            if (lc < nch) break;
            ++ls; lc = 0;
        }
        if (ls <= s_last) {
            const int b = blk(ls), b0 = b * TB, bs = min(TB, n - b0);
            const int r0 = ra + lc * RT, r1 = min(rb, r0 + RT);
            C *dst = tile + (size_t)(issued & 1) * RT * TRSV_TBP;
            if constexpr (sizeof(R) == 8) {                                 // 16 bytes a column: 64 threads a row
                const int q = threadIdx.x & 63;
                if (q < bs)
                    for (int r = threadIdx.x >> 6; r < r1 - r0; r += TRSV_NT / 64)
                        cp_async16(dst + (size_t)r * TRSV_TBP + q, Ac + (size_t)(r0 + r) * a.lda + b0 + q);
            } else if (vec16) {                                             // a warp a row: lane q copies 16 bytes
                const int q = threadIdx.x & 31;                             // (an odd last column alone, 8 bytes)
                if (2 * q < bs)
                    for (int r = threadIdx.x >> 5; r < r1 - r0; r += TRSV_NT / 32) {
                        const C *src = Ac + (size_t)(r0 + r) * a.lda + b0 + 2 * q;
                        if (2 * q + 1 < bs) cp_async16(dst + (size_t)r * TRSV_TBP + 2 * q, src);
                        else cp_async8(dst + (size_t)r * TRSV_TBP + 2 * q, src);
                    }
            } else {                                                        // 8 bytes a column: 64 threads a row
                const int q = threadIdx.x & 63;
                if (q < bs)
                    for (int r = threadIdx.x >> 6; r < r1 - r0; r += TRSV_NT / 64)
                        cp_async8(dst + (size_t)r * TRSV_TBP + q, Ac + (size_t)(r0 + r) * a.lda + b0 + q);
            }
            ++issued;
            ++lc;
        }
        cp_async_commit();                                                  // (an empty group past the last task)
    };
    // block b's inverse, transposed: Wt[rr][k] = W_b[k][rr] (W_b row-major TB x TB; 16-byte loads, one round trip)
    auto stage_w = [&](int b, C *dst) {
        const R *Wr = a.inv + 2 * ((size_t)b * 2 * TB * TB + (a.backward ? 0 : (size_t)TB * TB));
        if constexpr (sizeof(R) == 4) {
            const float4 *W = reinterpret_cast<const float4 *>(Wr);
            float4 v[TB * TB / 2 / TRSV_NT];
#pragma unroll
            for (int i = 0; i < TB * TB / 2 / TRSV_NT; ++i) v[i] = __ldg(W + threadIdx.x + TRSV_NT * i);
#pragma unroll
            for (int i = 0; i < TB * TB / 2 / TRSV_NT; ++i) {
                const int e = 2 * (threadIdx.x + TRSV_NT * i), k = e / TB, rr = e % TB;   // (k, rr), (k, rr + 1)
                dst[(size_t)rr * TRSV_TBP + k] = mk<float>(v[i].x, v[i].y);
                dst[(size_t)(rr + 1) * TRSV_TBP + k] = mk<float>(v[i].z, v[i].w);
            }
        } else {
            const double2 *W = reinterpret_cast<const double2 *>(Wr);
            double2 v[TB * TB / TRSV_NT];
#pragma unroll
            for (int i = 0; i < TB * TB / TRSV_NT; ++i) v[i] = __ldg(W + threadIdx.x + TRSV_NT * i);
#pragma unroll
            for (int i = 0; i < TB * TB / TRSV_NT; ++i) {
                const int e = threadIdx.x + TRSV_NT * i, k = e / TB, rr = e % TB;
                dst[(size_t)rr * TRSV_TBP + k] = mk<double>(v[i].x, v[i].y);
            }
        }
    };
    auto wbuf = [&](int b) { return Wt + (size_t)(nw == 1 ? 0 : b - bb0) * TB * TRSV_TBP; };
    if (nw == 1) stage_w(a.backward ? bb1 - 1 : bb0, Wt);                  // my first block's inverse
    else for (int b = bb0; b < bb1; ++b) stage_w(b, wbuf(b));               // both of mine
    issue_next();                                                           // task 0
    __syncthreads();
    int used = 0;
    for (int st = 0; st <= s_last; ++st) {
        const int b = blk(st), b0 = b * TB, bs = min(TB, n - b0);
        const bool mine = b >= bb0 && b < bb1;
        if (!mine) {
            if (threadIdx.x == 0) {
                long it = 0;
                while (ld_acquire_u32((const unsigned *)(a.flags + b)) != (unsigned)epoch) {
                    if ((++it & 1023) == 0 && (it > (1L << 21) || *(volatile int *)a.err)) {   // ~1 s
                        ok = 0; dev_error(a.err, M25_DEV_TIMEOUT); break;
                    }
                }
            }
            __syncthreads();
            if (!ok) { cp_async_wait0(); return; }
            {                                                               // another CTA's values: past L1,
                typedef typename vec2_of<R>::type V2;                       // all loads before the stores
                const V2 *p = reinterpret_cast<const V2 *>(a.Xout) + (size_t)b0 * nrhs;
                V2 v[TB * 16 / TRSV_NT];
#pragma unroll
                for (int i = 0; i < TB * 16 / TRSV_NT; ++i) {
                    const int e = threadIdx.x + TRSV_NT * i;
                    if (e < bs * nrhs) v[i] = __ldcg(p + e);
                }
#pragma unroll
                for (int i = 0; i < TB * 16 / TRSV_NT; ++i) {
                    const int e = threadIdx.x + TRSV_NT * i;
                    if (e < bs * nrhs) Yb[(e / nrhs) * TRSV_YS + e % nrhs] = mk<R>(v[i].x, v[i].y);
                }
            }
        } else {
            // every earlier block has been applied to this block's rows: y_b = W_b^T t_b
            tile_mul<KR, TRSV_NT / TB, false>(wbuf(b), bs, bs, T + (size_t)(b0 - R0) * TRSV_TS, TRSV_TS, Yb,
                                              TRSV_YS);
            __syncthreads();
            for (int e = threadIdx.x; e < bs * nrhs; e += blockDim.x)
                stc<R>(a.Xout, (size_t)b0 * nrhs + e, Yb[(e / nrhs) * TRSV_YS + e % nrhs]);
            __syncthreads();
            if (threadIdx.x == 0) {                                         // the CTA's stores, then the flag
                __threadfence();
                atomicExch(a.flags + b, epoch);
            }
            const int nxt = a.backward ? b - 1 : b + 1;                    // my next block's inverse (one buffer)
            if (nw == 1 && nxt >= bb0 && nxt < bb1) stage_w(nxt, Wt);
        }
        int ra, rb;
        rows_of(b, ra, rb);
        for (int r0 = ra; r0 < rb; r0 += RT) {
            issue_next();                                                   // the next task's tile, other buffer
            cp_async_wait1();                                               // this task's tile has landed
            __syncthreads();
            tile_mul<KR, TRSV_NT / RT, true>(tile + (size_t)(used & 1) * RT * TRSV_TBP, min(rb, r0 + RT) - r0, bs,
                                             Yb, TRSV_YS, T + (size_t)(r0 - R0) * TRSV_TS, TRSV_TS);
            ++used;
            __syncthreads();                                                // the buffer is the next copy's
        }
        __syncthreads();
    }
    cp_async_wait0();
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
    b += (2 + 2 * (size_t)G) * sizeof(unsigned) + 256;             // barrier, the panel's generations
    b += (2 * (size_t)G * (LL_REC + 4 * NB) + 2 * 4 * NB) * 8 + 256; // the flagged exchange records
    if (single) b += 2 * (m25_umma_workspace(n, NB) + 256);          // one a stream (look-ahead)
    (void)n;
    return b;
}

// The LU's two internal streams on the current device: a high-priority one for the panels and everything on the
// critical path, a low-priority one for the trailing update of the previous outer block, so that the next block's
// panels run while that update does (look-ahead); and the events between them. One set per host thread and device,
// created on the thread's first factorisation there (calls from different threads, e.g. concurrent requests on
// their own streams, do not share them; calls from one thread are ordered by it).
namespace {
struct LuStreams { cudaStream_t hi = nullptr, lo = nullptr; cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr}; };
thread_local LuStreams g_lu[64];

int lu_streams(LuStreams *out)
{
    int dev = -1;
    M25_CHECK(cudaGetDevice(&dev));
    M25_REQUIRE(dev >= 0 && dev < 64, "m25_getrf: device index above 63");
    LuStreams &L = g_lu[dev];
    if (!L.hi) {
        int least = 0, greatest = 0;
        M25_CHECK(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        M25_CHECK(cudaStreamCreateWithPriority(&L.hi, cudaStreamNonBlocking, greatest));
        M25_CHECK(cudaStreamCreateWithPriority(&L.lo, cudaStreamNonBlocking, least));
        for (auto &e : L.ev) M25_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    *out = L;
    return M25_OK;
}
}  // namespace

// ---- the LU's tile parameters by matrix size (set by the autotuner, mom25d_b200.tune) --------------------------------
// Two tables, complex64 and complex128, of entries (n, outer panel width, panel blocks); a factorisation of size n
// takes the entry nearest to n in log n. Without entries: NB2 and min(SMs, 32).
namespace {
struct LuTuning { int n, nb2, blocks; };
LuTuning g_tuning[2][32];
int g_ntuning[2] = {0, 0};
std::mutex g_tuning_mu;
}  // namespace

extern "C" int m25_set_lu_tuning(int single, const int *h_n, const int *h_nb2, const int *h_blocks, int count)
{
    M25_REQUIRE(count >= 0 && count <= 32 && (count == 0 || (h_n && h_nb2 && h_blocks)),
                "m25_set_lu_tuning: 0 to 32 entries");
    LuTuning t[32];
    for (int i = 0; i < count; ++i) {
        M25_REQUIRE(h_n[i] >= 1 && h_nb2[i] >= NB && h_nb2[i] <= NB2 && h_nb2[i] % NB == 0 && h_blocks[i] >= 1 &&
                    h_blocks[i] <= 4096, "m25_set_lu_tuning: n >= 1, nb2 a multiple of 64 up to 256, blocks >= 1");
        t[i] = LuTuning{h_n[i], h_nb2[i], h_blocks[i]};
    }
    std::sort(t, t + count, [](const LuTuning &a, const LuTuning &b) { return a.n < b.n; });
    std::lock_guard<std::mutex> lk(g_tuning_mu);
    const int w = single ? 1 : 0;
    std::copy(t, t + count, g_tuning[w]);
    g_ntuning[w] = count;
    return M25_OK;
}

// The parameters a factorisation of size n (complex64 when single) uses: the table's entry nearest in log n, else
// the defaults; M25_NB2 and M25_PANEL_BLOCKS in the environment override both.
extern "C" int m25_get_lu_tuning(int n, int single, int *nb2, int *blocks)
{
    int G = sm_count();
    if (G <= 0) G = 148;
    int b2 = NB2, gm = std::min(G, 32);
    {
        std::lock_guard<std::mutex> lk(g_tuning_mu);
        const int w = single ? 1 : 0;
        if (g_ntuning[w]) {
            int k = 0;
            double best = 1e300;
            for (int i = 0; i < g_ntuning[w]; ++i) {
                const double d = fabs(log((double)g_tuning[w][i].n / (double)std::max(1, n)));
                if (d < best) { best = d; k = i; }
            }
            b2 = g_tuning[w][k].nb2;
            gm = std::min(G, g_tuning[w][k].blocks);
        }
    }
    if (const char *e = getenv("M25_PANEL_BLOCKS")) gm = std::max(1, std::min(G, atoi(e)));
    if (const char *e = getenv("M25_NB2")) b2 = std::max(NB, std::min(NB2, atoi(e) / NB * NB));
    if (nb2) *nb2 = b2;
    if (blocks) *blocks = gm;
    return M25_OK;
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
    unsigned *bar = (unsigned *)take((2 + 2 * (size_t)G) * sizeof(unsigned));
    const size_t ll_bytes = (2 * (size_t)G * (LL_REC + 4 * NB) + 2 * 4 * NB) * 8;
    pw.ll_cand = (unsigned long long *)take(ll_bytes);
    pw.ll_row = pw.ll_cand + 2 * (size_t)G * LL_REC;
    pw.ll_drow = pw.ll_row + 2 * (size_t)G * 4 * NB;
    void *umma_work0 = take(0);
    size_t umma_bytes = (work_bytes - ((unsigned char *)umma_work0 - (unsigned char *)work)) / 2 / 256 * 256;
    void *umma_work1 = (unsigned char *)umma_work0 + umma_bytes;
    pw.bar.count = bar; pw.bar.gen = bar + 1;
    pw.gen = bar + 2;
    int *err = m25_dev_err_word();
    LuStreams st;
    int rc = lu_streams(&st);
    if (rc) return rc;
    const char *la = getenv("M25_LOOKAHEAD");                       // 0: one stream (the same results, in order)
    const cudaStream_t H = st.hi, Lo = (la && atoi(la) == 0) ? st.hi : st.lo;
    cudaEvent_t ev_start = st.ev[0], ev_panel = st.ev[1], ev_next = st.ev[2], ev_lo = st.ev[3], ev_end = st.ev[4];
    M25_CHECK(cudaEventRecord(ev_start, s));                        // the caller's work first
    M25_CHECK(cudaStreamWaitEvent(H, ev_start, 0));
    M25_CHECK(cudaStreamWaitEvent(Lo, ev_start, 0));
    M25_CHECK(cudaMemsetAsync(ipiv, 0xff, sizeof(int) * (size_t)n, H));      // -1 until the panel sets it
    M25_CHECK(cudaMemsetAsync(pw.ll_cand, 0, ll_bytes, H));         // flags 0: no column's (they are column + 1)
    const size_t trsm_smem = sizeof(cpx<R>) * (NB * NB + NB * 64);
    M25_CHECK(cudaFuncSetAttribute(k_trsm<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trsm_smem));
    M25_CHECK(cudaFuncSetAttribute(k_trsm64<R, t64_warps<R>(), false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)t64_smem<R>()));
    M25_CHECK(cudaFuncSetAttribute(k_trsm64<R, t64_warps<R>(), true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)t64_smem<R>()));
    M25_CHECK(cudaFuncSetAttribute(k_trsm_outer<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)to_smem<R>()));
    int smem_optin = 0, dev = 0;
    M25_CHECK(cudaGetDevice(&dev));
    M25_CHECK(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes pfa;
    M25_CHECK(cudaFuncGetAttributes(&pfa, k_panel_smem<R, false>));
    const int smem_cap = smem_optin - (int)pfa.sharedSizeBytes;      // less the kernel's static shared memory
    M25_CHECK(cudaFuncSetAttribute(k_panel_smem<R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_cap));
    // The cluster panel (the exchange in distributed shared memory) takes the panels whose rows fit a cluster's
    // blocks: as many blocks as the largest cluster this kernel can have on the device (16 where non-portable
    // sizes are allowed), a block's rows and its records in its shared memory. M25_PANEL_CLUSTER=0: never.
    int cl_max = 0, cl_rows_cap = 0;
    {
        const char *e = getenv("M25_PANEL_CLUSTER");
        if (!e || atoi(e) != 0) {
            cudaFuncAttributes cfa;
            M25_CHECK(cudaFuncGetAttributes(&cfa, k_panel_smem<R, true>));
            const int cl_smem = smem_optin - (int)cfa.sharedSizeBytes;
            M25_CHECK(cudaFuncSetAttribute(k_panel_smem<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, cl_smem));
            M25_CHECK(cudaFuncSetAttribute(k_panel_smem<R, true>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
            cl_rows_cap = (int)(((size_t)cl_smem - sizeof(PanelRecords) - 16) / (sizeof(cpx<R>) * NB));
            cudaLaunchConfig_t qc = {};
            cudaLaunchAttribute qa[1];
            qa[0].id = cudaLaunchAttributeClusterDimension;
            qa[0].val.clusterDim.x = 16; qa[0].val.clusterDim.y = 1; qa[0].val.clusterDim.z = 1;
            qc.gridDim = dim3(16); qc.blockDim = dim3(PANEL_THREADS); qc.dynamicSmemBytes = (size_t)cl_smem;
            qc.attrs = qa; qc.numAttrs = 1;
            int mc = 0;
            if (cudaOccupancyMaxPotentialClusterSize(&mc, (void *)k_panel_smem<R, true>, &qc) != cudaSuccess) {
                (void)cudaGetLastError();
                mc = 0;
            }
            cl_max = std::min(16, mc);
            if (const char *m = getenv("M25_PANEL_CLUSTER_MAX")) cl_max = std::min(cl_max, atoi(m));
            if (cl_max < 2) cl_max = 0;
        }
    }
    // Blocks of the panel: few enough that the cooperative launch finds its SMs quickly while the other stream's
    // update holds the rest (the exchange costs about the same from 37 to 148 blocks), but at least as many as
    // the panel's rows need to fit in shared memory (M25_PANEL_BLOCKS: tuning)
    int gmax = 32, nb2 = NB2;                                        // outer panel width and panel blocks: the
    m25_get_lu_tuning(n, sizeof(R) == 4, &nb2, &gmax);               // autotuner's table, else the defaults
    const int rows_cap = (int)((size_t)smem_cap / (sizeof(cpx<R>) * NB));   // a block's rows in shared memory
    const int gcap = std::min(G, PANEL_THREADS);                     // a thread of each block reads a block's record
    M25_CHECK(cudaFuncSetAttribute(k_gemm_update<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemm_smem<R>()));
    M25_CHECK(cudaFuncSetAttribute(k_zgemm_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zdmma_smem()));
    // the interchanges ipiv[r0 .. r0 + nsw) on the columns [a0, a1) and [b0, b1); groups > 1: group g takes the
    // rows, count and first range shifted by g gs
    auto laswp = [&](int r0, int nsw, long a0, long a1, long b0, long b1, int gs, int groups, cudaStream_t cs) -> int {
        const long nc = std::max(0L, a1 - a0) + std::max(0L, b1 - b0);
        if (nc <= 0 || nsw <= 0) return M25_OK;
        const long bx = std::min<long>((nc + 15) / 16, 4L * G);
        k_laswp_plan<R><<<dim3((unsigned)bx, (unsigned)groups), 256, 0, cs>>>(A, lda, n, ipiv, r0, nsw, a0,
                                                                             std::max(a0, a1), b0, std::max(b0, b1),
                                                                             gs, err);
        M25_LAUNCH_CHECK("k_laswp_plan");
        return M25_OK;
    };
    // U12 rows k0 .. k0 + jb of the columns [c0, c1); swap: the panel's interchanges applied to them on the way
    auto trsm = [&](int k0, int jb, long c0, long c1, bool swap, cudaStream_t cs) -> int {
        if (c1 <= c0) return M25_OK;
        if (jb == NB) {
            const long per = 32L * t64_warps<R>();
            const unsigned grid = (unsigned)((c1 - c0 + per - 1) / per);
            if (swap)
                k_trsm64<R, t64_warps<R>(), true><<<grid, (unsigned)per, t64_smem<R>(), cs>>>(A, lda, k0, c0, c1,
                                                                                               ipiv, n, err);
            else
                k_trsm64<R, t64_warps<R>(), false><<<grid, (unsigned)per, t64_smem<R>(), cs>>>(A, lda, k0, c0, c1,
                                                                                                ipiv, n, err);
            M25_LAUNCH_CHECK("k_trsm64");
            return M25_OK;
        }
        int rc2;
        if (swap && (rc2 = laswp(k0, jb, c0, c1, 0, 0, 0, 1, cs))) return rc2;
        k_trsm<R><<<(c1 - c0 + 63) / 64, 256, trsm_smem, cs>>>(A, lda, k0, jb, c0, c1);
        M25_LAUNCH_CHECK("k_trsm");
        return M25_OK;
    };
    // U12 of the whole outer panel [K0, K0 + JB) on the columns [c0, c1), its interchanges applied on the way
    auto trsm_outer = [&](int K0, int JB, long c0, long c1, cudaStream_t cs) -> int {
        if (c1 <= c0) return M25_OK;
        k_trsm_outer<R><<<(unsigned)((c1 - c0 + TO_COLS - 1) / TO_COLS), TO_THREADS, to_smem<R>(), cs>>>(
            A, lda, n, K0, JB, ipiv, c0, c1, err);
        M25_LAUNCH_CHECK("k_trsm_outer");
        return M25_OK;
    };
    // C = A[r0 .., c0 ..] (M x Nc) -= A[r0 .., k0 .. k0 + K] A[k0 .. k0 + K, c0 ..]; the low-priority stream's
    // tensor-core updates split their operands into the second workspace
    auto gemm = [&](int r0, int M, long c0, int Nc, int k0, int K, bool big, cudaStream_t cs) -> int {
        if (M <= 0 || Nc <= 0 || K <= 0) return M25_OK;
        R *C22 = A + 2 * ((size_t)c0 * lda + r0);
        const R *L21 = A + 2 * ((size_t)k0 * lda + r0);
        const R *U12 = A + 2 * ((size_t)c0 * lda + k0);
        if (sizeof(R) == 4 && tf32 && big)
            return m25_umma_trailing((float *)C22, lda, M, Nc, K, (const float *)L21, (const float *)U12,
                                     cs == Lo ? umma_work1 : umma_work0, umma_bytes, cs);
        if (sizeof(R) == 8) {                                      // complex128: the FP64 tensor cores
            dim3 grid((Nc + ZD_BN - 1) / ZD_BN, (M + ZD_BM - 1) / ZD_BM);
            k_zgemm_dmma<<<grid, 128, zdmma_smem(), cs>>>((double *)C22, (const double *)L21, (const double *)U12,
                                                          lda, M, Nc, K);
            M25_LAUNCH_CHECK("k_zgemm_dmma");
            return M25_OK;
        }
        dim3 grid((Nc + 63) / 64, (M + 127) / 128);
        k_gemm_update<R><<<grid, 256, gemm_smem<R>(), cs>>>(C22, L21, U12, lda, M, Nc, K);
        M25_LAUNCH_CHECK("k_gemm_update");
        return M25_OK;
    };
    // Two levels: outer panels of nb2 columns, each factored as panels of NB (pivoting, interchanges, TRSM and
    // updates restricted to the outer panel). Then, for outer block k of columns [K0, KE), the next block's columns
    // [KE, KE2) and the rest [KE2, n):
    //   H (high priority, the critical path): the next block's interchanges, U12 and update by block k, then the
    //     next block's panels. Before touching those columns it waits only for the part of the previous block's
    //     low-priority update that covers them (ev_next), which that update does first;
    //   Lo (low priority): as soon as block k's panels are done (ev_panel), block k's interchanges on the columns
    //     left of it and on [KE2, n), U12 of [KE2, n), then the update of [KE2, n): first the columns of block
    //     k + 2 ([KE2, KE3): ev_next, which H waits for at block k + 1), then the rest.
    // Regions: H works on columns >= KE only; Lo on columns < K0 (interchanges) and >= KE2; both read block k's
    // L (rows >= KE of columns [K0, KE)), which nothing writes until block k + 1's left interchanges, issued on Lo
    // after this update. Lo's work for a block follows its work for the previous block (stream order).
    bool next_pending = false;
    for (int K0 = 0; K0 < n; K0 += nb2) {
        const int JB = std::min(nb2, n - K0), KE = K0 + JB;
        const int KE2 = std::min(n, KE + nb2), KE3 = std::min(n, KE2 + nb2);
        for (int k0 = K0; k0 < KE; k0 += NB) {
            const int jb = std::min(NB, KE - k0);
            int Gp = std::min(gmax, std::max(1, (n - k0 + 31) / 32));
            Gp = std::min(gcap, std::max(Gp, (n - k0 + rows_cap - 1) / rows_cap));
            const int cs = (n - k0 + Gp - 1) / Gp;
            const size_t psmem = sizeof(cpx<R>) * (size_t)cs * jb;
            void *args[] = {&A, &lda, &n, (void *)&k0, (void *)&jb, &ipiv, &pw, &err};
            const int rows = n - k0;
            if (cl_max && rows <= cl_max * cl_rows_cap) {               // one cluster, at least 64 rows a block
                const int Gc = std::min(cl_max, std::max(2, (rows + 63) / 64));
                const int csc = (rows + Gc - 1) / Gc;
                cudaLaunchConfig_t lc = {};
                cudaLaunchAttribute la1[1];
                la1[0].id = cudaLaunchAttributeClusterDimension;
                la1[0].val.clusterDim.x = (unsigned)Gc; la1[0].val.clusterDim.y = 1; la1[0].val.clusterDim.z = 1;
                lc.gridDim = dim3(Gc); lc.blockDim = dim3(PANEL_THREADS);
                lc.dynamicSmemBytes = ((size_t)csc * jb * sizeof(cpx<R>) + 15) / 16 * 16 + sizeof(PanelRecords);
                lc.stream = H; lc.attrs = la1; lc.numAttrs = 1;
                M25_CHECK(cudaLaunchKernelExC(&lc, (const void *)k_panel_smem<R, true>, args));
            } else if (psmem <= (size_t)smem_cap) {                    // (flagged records: no barrier to reset)
                M25_CHECK(cudaLaunchCooperativeKernel((void *)k_panel_smem<R, false>, dim3(Gp), dim3(PANEL_THREADS),
                                                      args, psmem, H));
            } else {
                M25_CHECK(cudaMemsetAsync(bar, 0, (2 + 2 * (size_t)G) * sizeof(unsigned), H));
                M25_CHECK(cudaLaunchCooperativeKernel((void *)k_panel<R>, dim3(Gp), dim3(PANEL_THREADS), args, 0, H));
            }
            m25_note_launch();
            if ((rc = trsm(k0, jb, k0 + jb, KE, true, H))) return rc;     // the rest of the outer panel
            // in FP32 on the CUDA cores, not 3xTF32: the columns of L pass through every update of their outer
            // panel, and the tensor-core error there (about 2^-22 a product against 2^-24) costs the factor its
            // use as a preconditioner near the low-frequency end (fresh LUs at 0.67 and 0.91 GHz of the routed
            // board no longer converged; the FP32 inner update costs 5 ms of 236 at N = 18,788)
            if ((rc = gemm(k0 + jb, n - k0 - jb, k0 + jb, KE - k0 - jb, k0, jb, false, H))) return rc;
        }
        // each earlier panel's columns of the outer panel: the interchanges of the panels after it (one launch)
        const int npan = (JB + NB - 1) / NB;
        if (npan > 1 && (rc = laswp(K0 + NB, JB - NB, K0, K0 + NB, 0, 0, NB, npan - 1, H))) return rc;
        M25_CHECK(cudaEventRecord(ev_panel, H));                          // block k's L and pivots are final
        if (KE < n) {                                                       // H: the next block's columns
            if (next_pending) M25_CHECK(cudaStreamWaitEvent(H, ev_next, 0));
            if ((rc = trsm_outer(K0, JB, KE, KE2, H))) return rc;          // interchanges and U12 in one launch
            if ((rc = gemm(KE, n - KE, KE, KE2 - KE, K0, JB, true, H))) return rc;
        }
        M25_CHECK(cudaStreamWaitEvent(Lo, ev_panel, 0));                    // Lo: the left and the far columns
        if ((rc = laswp(K0, JB, 0, K0, KE2, n, 0, 1, Lo))) return rc;      // (one launch for both)
        next_pending = false;
        if (KE2 < n) {
            for (int k0 = K0; k0 < KE; k0 += NB) {
                const int jb = std::min(NB, KE - k0);
                if ((rc = trsm(k0, jb, KE2, n, false, Lo))) return rc;
                if ((rc = gemm(k0 + jb, KE - k0 - jb, KE2, n - KE2, k0, jb, true, Lo))) return rc;
            }
            if ((rc = gemm(KE, n - KE, KE2, KE3 - KE2, K0, JB, true, Lo))) return rc;   // block k + 2's columns
            M25_CHECK(cudaEventRecord(ev_next, Lo));
            next_pending = true;
            if ((rc = gemm(KE, n - KE, KE3, n - KE3, K0, JB, true, Lo))) return rc;    // the rest
        }
    }
    M25_CHECK(cudaEventRecord(ev_lo, Lo));                           // the last left interchanges, then the end
    M25_CHECK(cudaStreamWaitEvent(H, ev_lo, 0));
    M25_CHECK(cudaEventRecord(ev_end, H));                           // the caller's stream waits for both
    M25_CHECK(cudaStreamWaitEvent(s, ev_end, 0));
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
static size_t aux_layout(int n, size_t *off_inv, size_t *off_perm, size_t *off_w, size_t *off_flags = nullptr)
{
    const size_t nb = (n + TB - 1) / TB;
    size_t o = 0;
    *off_inv = o; o += nb * 2 * TB * TB * sizeof(cpx<R>); o = (o + 255) / 256 * 256;
    *off_perm = o; o += sizeof(int) * (size_t)n; o = (o + 255) / 256 * 256;
    *off_w = o; o += 2 * (size_t)n * 16 * sizeof(cpx<R>); o = (o + 255) / 256 * 256;
    if (off_flags) *off_flags = o;
    o += sizeof(int) * (2 * nb + 32);                  // flags of the two solves, then the epoch counter
    return o;
}

// The 256-row-block solves (trsv_sb.cu): their data after the 64-row-block solves' in the same aux buffer
bool m25_sb_enabled(int n, int single);
size_t m25_sb_bytes(int n, int single);
int m25_sb_prepare(const void *A, long lda, int n, int single, const void *inv64, void *sb, cudaStream_t s);
int m25_sb_solve(const void *A, long lda, int n, int single, void *sb, const void *Tin, void *Xout, int nrhs,
                 int backward, const int *epoch, int *err, cudaStream_t s);

// the 64-row-block solves' data alone (the layout of m25_getrs_noalloc's fixed scratch)
size_t m25_getrs_aux_bytes_basic(int n, int single)
{
    size_t a, b, c;
    return single ? aux_layout<float>(n, &a, &b, &c) : aux_layout<double>(n, &a, &b, &c);
}
// where the 256-row-block solves' data starts in an aux buffer
static size_t sb_offset(int n, int single) { return (m25_getrs_aux_bytes_basic(n, single) + 255) / 256 * 256; }

extern "C" size_t m25_getrs_aux_bytes(int n, int single)
{
    const size_t sb = m25_sb_bytes(n, single);
    return sb ? sb_offset(n, single) + sb : m25_getrs_aux_bytes_basic(n, single);
}

template <typename R>
static size_t trsv_smem(int n, int G)
{
    const int nb = (n + TB - 1) / TB, per = (nb + G - 1) / G;
    return sizeof(cpx<R>) * (TB * (TB + 1) + TB * 16 + (size_t)per * TB * 16);
}

// sb: the 256-row-block solves where m25_sb_enabled (their data after the basic layout); false keeps the basic
// layout alone (m25_getrs_noalloc's fixed scratch)
template <typename R>
static int getrs_prepare_impl(const R *A, long lda, int n, const int *ipiv, unsigned char *aux, size_t aux_bytes,
                              cudaStream_t s, bool sb)
{
    size_t oi, op, ow, of;
    M25_REQUIRE(aux_bytes >= aux_layout<R>(n, &oi, &op, &ow, &of), "m25_getrs_prepare: aux buffer too small");
    const int single = sizeof(R) == 4;
    const bool use_sb = sb && m25_sb_enabled(n, single);
    const size_t basic = sb_offset(n, single);
    if (use_sb) M25_REQUIRE(aux_bytes >= basic + m25_sb_bytes(n, single), "m25_getrs_prepare: aux buffer too small");
    const int nb = (n + TB - 1) / TB;
    const size_t ismem = 2 * sizeof(cpx<R>) * TB * (TB + 1);
    M25_CHECK(cudaFuncSetAttribute(k_block_inverses<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ismem));
    k_block_inverses<R><<<nb, TB, ismem, s>>>(A, lda, n, (R *)(aux + oi));
    M25_LAUNCH_CHECK("k_block_inverses");
    M25_REQUIRE(sizeof(int) * (size_t)n <= 200 * 1024, "m25_getrs_prepare: n above 51200");
    M25_CHECK(cudaFuncSetAttribute(k_perm_from_ipiv, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(sizeof(int) * n)));
    k_perm_from_ipiv<<<1, 1024, sizeof(int) * n, s>>>(ipiv, n, (int *)(aux + op));
    M25_LAUNCH_CHECK("k_perm_from_ipiv");
    M25_CHECK(cudaMemsetAsync(aux + of, 0, sizeof(int) * (2 * nb + 32), s));
    if (use_sb) return m25_sb_prepare(A, lda, n, single, aux + oi, aux + basic, s);
    return M25_OK;
}

template <typename R>
static int getrs_aux_impl(const R *A, long lda, int n, unsigned char *aux, R *B, int nrhs, cudaStream_t s, int *err,
                          bool sb)
{
    size_t oi, op, ow, of;
    aux_layout<R>(n, &oi, &op, &ow, &of);
    const R *inv = (const R *)(aux + oi);
    const int *perm = (const int *)(aux + op);
    R *W1 = (R *)(aux + ow), *W2 = W1 + 2 * (size_t)n * 16;
    const int nb = (n + TB - 1) / TB;
    int *flags = (int *)(aux + of), *epoch = flags + 2 * nb;
    const int single = sizeof(R) == 4;
    if (sb && nrhs <= 8 && m25_sb_enabled(n, single)) {
        // 256-row diagonal blocks, the chain between blocks one product a block (trsv_sb.cu)
        unsigned char *sbd = aux + sb_offset(n, single);
        k_bump_epoch<<<1, 1, 0, s>>>(epoch);
        M25_LAUNCH_CHECK("k_bump_epoch");
        int rc = m25_sb_solve(A, lda, n, single, sbd, B, W1, nrhs, 0, epoch, err, s);   // U^T y = b
        if (!rc) rc = m25_sb_solve(A, lda, n, single, sbd, W1, W2, nrhs, 1, epoch, err, s);   // L^T z = y
        if (rc) return rc;
        long tot = (long)n * nrhs;                                          // X = P z
        k_gather_rows<R><<<(tot + 255) / 256, 256, 0, s>>>(W2, B, perm, n, nrhs);
        M25_LAUNCH_CHECK("k_gather_rows");
        return M25_OK;
    }
    // CTAs of the persistent solves: one an SM (measured at N = 18,788, complex64, 8 columns: 3.4 ms with 148 CTAs,
    // 4.8 / 5.3 / 6.6 ms with 100 / 74 / 59, each owning more consecutive blocks)
    const int G = std::max(1, std::min(sm_count(), nb));
    const size_t sm = trsv_smem<R>(n, G);
    M25_REQUIRE(sm <= 200 * 1024, "m25_getrs_aux: n too large for the persistent solve");
    M25_CHECK(cudaFuncSetAttribute(k_trsv_persistent<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_bump_epoch<<<1, 1, 0, s>>>(epoch);                                    // this call's flag value
    M25_LAUNCH_CHECK("k_bump_epoch");
    TrsvArgs<R> fa{A, lda, n, nb, inv, B, W1, nrhs, 0, flags, epoch, err};          // U^T y = b: B -> W1
    TrsvArgs<R> ba{A, lda, n, nb, inv, W1, W2, nrhs, 1, flags + nb, epoch, err};    // L^T z = y: W1 -> W2
    const int per = (nb + G - 1) / G;
    int smem_optin = 0, dev = 0;
    M25_CHECK(cudaGetDevice(&dev));
    M25_CHECK(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (per <= TRSV_MAXPER && trsv_pipe_smem<R>(per) + 256 <= (size_t)smem_optin) {
        // the factor tiles through shared memory (cp.async, 16-byte pieces where rows allow); the kernel for the
        // smallest compile-time column count >= nrhs
        const size_t psm = trsv_pipe_smem<R>(per);
        int vec16 = (lda % 2 == 0) && (reinterpret_cast<uintptr_t>(A) % 16 == 0);
        const void *kf = nrhs <= 1 ? (const void *)k_trsv_pipe<R, 1> : nrhs <= 2 ? (const void *)k_trsv_pipe<R, 2> :
                         nrhs <= 4 ? (const void *)k_trsv_pipe<R, 4> : nrhs <= 8 ? (const void *)k_trsv_pipe<R, 8> :
                         (const void *)k_trsv_pipe<R, 16>;
        M25_CHECK(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm));
        void *fargs[] = {&fa, &vec16};
        M25_CHECK(cudaLaunchCooperativeKernel(kf, dim3(G), dim3(TRSV_NT), fargs, psm, s));
        m25_note_launch();
        void *bargs[] = {&ba, &vec16};
        M25_CHECK(cudaLaunchCooperativeKernel(kf, dim3(G), dim3(TRSV_NT), bargs, psm, s));
        m25_note_launch();
    } else {
        void *fargs[] = {&fa};
        M25_CHECK(cudaLaunchCooperativeKernel((void *)k_trsv_persistent<R>, dim3(G), dim3(256), fargs, sm, s));
        m25_note_launch();
        void *bargs[] = {&ba};
        M25_CHECK(cudaLaunchCooperativeKernel((void *)k_trsv_persistent<R>, dim3(G), dim3(256), bargs, sm, s));
        m25_note_launch();
    }
    long tot = (long)n * nrhs;                                              // X = P z
    k_gather_rows<R><<<(tot + 255) / 256, 256, 0, s>>>(W2, B, perm, n, nrhs);
    M25_LAUNCH_CHECK("k_gather_rows");
    return M25_OK;
}

extern "C" int m25_getrs_prepare(const void *d_LU, long lda, int n, const int *d_ipiv, int single, void *d_aux,
                                 size_t aux_bytes, void *stream)
{
    M25_REQUIRE(d_LU && d_ipiv && d_aux && n >= 1 && lda >= n, "m25_getrs_prepare: LU, ipiv, aux, n >= 1");
    return single ? getrs_prepare_impl<float>((const float *)d_LU, lda, n, d_ipiv, (unsigned char *)d_aux, aux_bytes,
                                              S(stream), true)
                  : getrs_prepare_impl<double>((const double *)d_LU, lda, n, d_ipiv, (unsigned char *)d_aux, aux_bytes,
                                               S(stream), true);
}

extern "C" int m25_getrs_aux(const void *d_LU, long lda, int n, int single, void *d_aux, void *d_B, int nrhs, void *stream)
{
    M25_REQUIRE(d_LU && d_aux && d_B && n >= 1 && lda >= n, "m25_getrs_aux: LU, aux, B, n >= 1");
    M25_REQUIRE(nrhs >= 1 && nrhs <= 16, "m25_getrs_aux: 1 to 16 right-hand sides a call");
    int *err = m25_dev_err_word();
    return single ? getrs_aux_impl<float>((const float *)d_LU, lda, n, (unsigned char *)d_aux, (float *)d_B, nrhs, S(stream),
                                          err, true)
                  : getrs_aux_impl<double>((const double *)d_LU, lda, n, (unsigned char *)d_aux, (double *)d_B, nrhs,
                                           S(stream), err, true);
}

extern "C" int m25_getrs(const void *d_LU, long lda, int n, const int *d_ipiv, int single, void *d_B, int nrhs, void *stream)
{
    M25_REQUIRE(d_LU && d_ipiv && d_B && n >= 1 && lda >= n, "m25_getrs: LU, ipiv, B, n >= 1");
    M25_REQUIRE(nrhs >= 1 && nrhs <= 16, "m25_getrs: 1 to 16 right-hand sides a call");
    // one call: by 64-row diagonal blocks (the 256-row blocks' inverses and couplings pay off only over many solves
    // with one factor, m25_getrs_prepare / m25_getrs_aux)
    const size_t bytes = m25_getrs_aux_bytes_basic(n, single);
    void *aux = nullptr;
    M25_CHECK(cudaMallocAsync(&aux, bytes, S(stream)));
    int *err = m25_dev_err_word();
    int rc = single ? getrs_prepare_impl<float>((const float *)d_LU, lda, n, d_ipiv, (unsigned char *)aux, bytes,
                                                S(stream), false)
                    : getrs_prepare_impl<double>((const double *)d_LU, lda, n, d_ipiv, (unsigned char *)aux, bytes,
                                                 S(stream), false);
    if (!rc)
        rc = single ? getrs_aux_impl<float>((const float *)d_LU, lda, n, (unsigned char *)aux, (float *)d_B, nrhs,
                                            S(stream), err, false)
                    : getrs_aux_impl<double>((const double *)d_LU, lda, n, (unsigned char *)aux, (double *)d_B, nrhs,
                                             S(stream), err, false);
    cudaError_t fe = cudaFreeAsync(aux, S(stream));
    if (!rc && fe != cudaSuccess) return m25_cuda_status(fe, "cudaFreeAsync");
    return rc;
}

// The solves of m25_getrs on caller-given scratch (aux_bytes >= m25_getrs_aux_bytes) with the device status word
// err: used by m25_getrs_noalloc, whose scratch and status word are file-scope device memory.
int m25_getrs_on_scratch(const void *d_LU, long lda, int n, const int *d_ipiv, int single, void *d_aux,
                         size_t aux_bytes, int *d_err, void *d_B, int nrhs, cudaStream_t s)
{
    int rc = single ? getrs_prepare_impl<float>((const float *)d_LU, lda, n, d_ipiv, (unsigned char *)d_aux, aux_bytes,
                                                s, false)
                    : getrs_prepare_impl<double>((const double *)d_LU, lda, n, d_ipiv, (unsigned char *)d_aux,
                                                 aux_bytes, s, false);
    if (rc) return rc;
    return single ? getrs_aux_impl<float>((const float *)d_LU, lda, n, (unsigned char *)d_aux, (float *)d_B, nrhs, s,
                                          d_err, false)
                  : getrs_aux_impl<double>((const double *)d_LU, lda, n, (unsigned char *)d_aux, (double *)d_B, nrhs,
                                           s, d_err, false);
}
