// umma.cu - the complex64 LU's trailing update C -= L U on the 5th-generation tensor cores (tcgen05), 3xTF32.
//
// Complex as real: with C, L, U column-major complex (interleaved re, im), C viewed as real is C' (2M x N) and
//   C' = A' B',  A' (2M x 2K): rows 2m, 2m+1 = [Lr -Li ; Li Lr] per k,   B' (2K x N): U's memory read as real.
// A' is built once per update (k_split_A), B' is U (k_split_B); both split into TF32 hi and lo parts
// (hi = rna(x), lo = x - hi) and D = lo_A hi_B + hi_A lo_B + hi_A hi_B accumulates in FP32 in tensor memory
// (3xTF32: the FP32 product to a few ulps). The 8/3 N^3 count of the LU is unchanged by the split.
//
// Kernel (one CTA per 128 x 256 tile of C', 4 warps):
//   warp 0 lane 0   TMA producer: per K stage of 32 floats, 4 tiled loads (A'hi, A'lo: 128 x 128 B; B'hi, B'lo:
//                   256 x 128 B; 128B swizzle) into one of two stages, completion on an mbarrier (complete_tx)
//   warp 1 lane 0   MMA issuer: 4 k-steps x 3 tcgen05.mma (M 128, N 256, K 8) per stage, tcgen05.commit frees
//                   the stage; the last commit signals the epilogue
//   warps 0-3       epilogue: tcgen05.ld of their 32 accumulator lanes, C -= D, coalesced along the column
// Every wait is bounded: on time-out the kernel records M25_DEV_TIMEOUT, waits (bounded) for the MMAs it issued,
// frees its tensor memory and returns. No multicast anywhere (single-GPU code, one CTA per cluster).
#include <cuda.h>
#include <algorithm>
#include <cstdlib>

#include "common.cuh"

int *m25_dev_err_word();

namespace {

// tile of C' (rows x cols), BKF floats of K per stage. Two stages of 16 floats (64-byte rows, 64B swizzle): 48 KB a
// stage, 97 KB a CTA, so two CTAs fit an SM (2 x 256 tensor-memory columns) and one's epilogue (C read, updated and
// written back) runs while the other multiplies, which one CTA with four stages could not do (3.92 -> 3.38 ms for an
// 18,000 x 18,000 x 256 complex update). Measured and not kept: four stages of 8 floats (32-byte rows, the same
// 97 KB): 4.23 ms, the tensor pipe 40% busy against 64% (smaller TMA boxes, a commit every three MMAs).
#ifndef M25_UMMA_BKF
#define M25_UMMA_BKF 16
#endif
#ifndef M25_UMMA_STAGES
#define M25_UMMA_STAGES 2
#endif
constexpr int BM = 128, BN = 256, BKF = M25_UMMA_BKF;
constexpr int STAGES = M25_UMMA_STAGES;
constexpr int RASTER = 16;                           // row tiles a group of the tile order
constexpr int SWZ_BYTES = BKF * 4;                   // the swizzle span: one K row of a stage
static_assert(SWZ_BYTES == 32 || SWZ_BYTES == 64 || SWZ_BYTES == 128, "32B, 64B or 128B swizzle");
constexpr int A_BYTES = BM * BKF * 4, B_BYTES = BN * BKF * 4;
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;          // hi and lo of A' and B'
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;   // + alignment slack + barriers
constexpr int CTAS_PER_SM = 2 * SMEM_BYTES <= 226 * 1024 ? 2 : 1;   // two CTAs an SM when their stages fit twice
static_assert(STAGE_BYTES % 1024 == 0, "stages on 1024-byte boundaries (swizzle atoms)");
constexpr unsigned TMEM_COLS = 256;
constexpr long WAIT_LIMIT = 1L << 24;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, unsigned parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}
// bounded wait: false if it gave up (or another thread of the CTA gave up)
__device__ __forceinline__ bool mbar_wait(uint32_t bar, unsigned parity, volatile int *abort)
{
    for (long it = 0; it < WAIT_LIMIT; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*abort) return false;
    }
    *abort = 1;
    return false;
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                 ::"r"(dst), "l"(map), "r"(x), "r"(y), "r"(bar) : "memory");
}

// shared-memory matrix descriptor: K-major, swizzled rows of SWZ_BYTES, 8-row groups 8 x SWZ_BYTES apart
// (tcgen05 layout, version 1; layout type 2 = 128B swizzle, 4 = 64B swizzle, 6 = 32B swizzle)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr & 0x3FFFF) >> 4);
    d |= (uint64_t)(16 >> 4) << 16;          // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)((8 * SWZ_BYTES) >> 4) << 32;   // stride byte offset
    d |= (uint64_t)1 << 46;                  // descriptor version
    d |= (uint64_t)(SWZ_BYTES == 128 ? 2 : SWZ_BYTES == 64 ? 4 : 6) << 61;
    return d;
}

// instruction descriptor: D F32, A and B TF32, both K-major, N = 256, M = 128
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
                 ::"r"(tmem_d), "l"(a), "l"(b), "r"(IDESC), "r"(accumulate) : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ float tf32_rna(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

__global__ void __launch_bounds__(128, CTAS_PER_SM) k_umma_update(float *C, long ldc_f, int Mp, int Nc, int kchunks,
                                                        const __grid_constant__ CUtensorMap mAhi,
                                                        const __grid_constant__ CUtensorMap mAlo,
                                                        const __grid_constant__ CUtensorMap mBhi,
                                                        const __grid_constant__ CUtensorMap mBlo, int *err)
{
    extern __shared__ unsigned char smem_raw[];
    const uint32_t base_raw = smem_u32(smem_raw);
    const uint32_t base = (base_raw + 1023) & ~1023u;              // 1024-aligned stages (swizzle atoms)
    const uint32_t bars = base + STAGES * STAGE_BYTES;
    // barriers: full[s] at bars + 8 s, empty[s] at bars + 16 + 8 s, done at bars + 32; tmem slot at bars + 40
    const uint32_t full0 = bars, empty0 = bars + 8 * STAGES, done = bars + 16 * STAGES;
    unsigned char *gen_bars = smem_raw + (bars - base_raw);
    volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(gen_bars + 16 * STAGES + 8);
    __shared__ int abort_flag;
    __shared__ int issued_k, consumed_k;                           // stages loaded / multiplied (abort clean-up)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // tile order: CTAs in launch order walk down a group of RASTER row tiles, then on to the next column tile, so the
    // CTAs in flight (two an SM) cover a block of about RASTER x 18 tiles whose A' and B' slabs stay in L2; in plain
    // order they swept every column tile of a row tile and read B' from DRAM again for every few row tiles
    int m0, n0;
    {
        const int nm = gridDim.y, nn = gridDim.x;
        const int pid = blockIdx.y * nn + blockIdx.x;
        const int group = pid / (RASTER * nn), first = group * RASTER;
        const int rows = min(nm - first, RASTER);
        const int in_group = pid - group * RASTER * nn;
        m0 = (first + in_group % rows) * BM;
        n0 = (in_group / rows) * BN;
    }

    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int s = 0; s < STAGES; ++s) { mbar_init(full0 + 8 * s, 1); mbar_init(empty0 + 8 * s, 1); }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issued_k = 0;
        consumed_k = 0;
    }
    __syncwarp();                                                   // (alloc is .sync.aligned: a converged warp)
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32((const void *)tmem_slot)), "r"(TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    volatile int *abort = &abort_flag;

    if (warp == 0 && lane == 0) {
        // producer
        for (int kc = 0; kc < kchunks; ++kc) {
            const int s = kc % STAGES;
            if (kc >= STAGES && !mbar_wait(empty0 + 8 * s, ((kc / STAGES) - 1) & 1, abort)) break;
            const uint32_t st = base + s * STAGE_BYTES;
            mbar_expect_tx(full0 + 8 * s, STAGE_BYTES);
            const int x = kc * BKF;
            tma_load_2d(st, &mAhi, x, m0, full0 + 8 * s);
            tma_load_2d(st + A_BYTES, &mAlo, x, m0, full0 + 8 * s);
            tma_load_2d(st + 2 * A_BYTES, &mBhi, x, n0, full0 + 8 * s);
            tma_load_2d(st + 2 * A_BYTES + B_BYTES, &mBlo, x, n0, full0 + 8 * s);
            issued_k = kc + 1;
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        int issued = 0;
        for (int kc = 0; kc < kchunks; ++kc) {
            const int s = kc % STAGES;
            if (!mbar_wait(full0 + 8 * s, (kc / STAGES) & 1, abort)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t st = base + s * STAGE_BYTES;
            const uint32_t aH = st, aL = st + A_BYTES, bH = st + 2 * A_BYTES, bL = st + 2 * A_BYTES + B_BYTES;
#pragma unroll
            for (int k = 0; k < BKF / 8; ++k) {
                const uint32_t off = k * 32;                     // 8 tf32 = 32 bytes along K inside the swizzle atom
                umma_tf32(tmem, sdesc(aL + off), sdesc(bH + off), issued > 0 ? 1u : 0u);
                umma_tf32(tmem, sdesc(aH + off), sdesc(bL + off), 1u);
                umma_tf32(tmem, sdesc(aH + off), sdesc(bH + off), 1u);
                ++issued;
            }
            umma_commit(empty0 + 8 * s);
            consumed_k = kc + 1;
        }
        umma_commit(done);                                   // (arrives once every MMA issued so far is complete)
    }
    __syncwarp();
    // epilogue: all four warps, warp w owns accumulator lanes 32 w .. 32 w + 31
    const bool ok = mbar_wait(done, 0, abort);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const bool go = __all_sync(0xffffffffu, ok && !*abort);        // warp-uniform: tcgen05.ld is .sync.aligned
    if (go) {
        const int row = m0 + warp * 32 + lane;
        for (int c0 = 0; c0 < BN; c0 += 32) {
            uint32_t v[32];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                         "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                           "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                           "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                           "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                           "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                         : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < Mp) {
                // all 32 loads issued before any store (a load -> store chain per column serialised the memory
                // latency 256 times a tile)
                float cv[32];
                float *p = C + (size_t)(n0 + c0) * ldc_f + row;
                const int nv = min(32, Nc - (n0 + c0));
#pragma unroll
                for (int j = 0; j < 32; ++j) cv[j] = j < nv ? __ldcs(p + (size_t)j * ldc_f) : 0.f;
#pragma unroll
                for (int j = 0; j < 32; ++j)    // (streaming: C is read and written once, the operands stay in L2)
                    if (j < nv) __stcs(p + (size_t)j * ldc_f, cv[j] - __uint_as_float(v[j]));
            }
        }
    }
    __syncthreads();
    if (*abort && threadIdx.x == 0) {
        dev_error(err, M25_DEV_TIMEOUT);
        // loads still in flight would land in this CTA's shared memory after it exits: wait for them (bounded)
        volatile int never = 0;
        for (int kc = consumed_k; kc < issued_k; ++kc) mbar_wait(full0 + 8 * (kc % STAGES), (kc / STAGES) & 1, &never);
        never = 0;
        mbar_wait(done, 0, &never);                          // and the MMAs issued (they read shared, write tensor memory)
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

// ---- the same update with a short run of tiles a CTA and two tensor-memory accumulators --------------------------
// One CTA an SM (four 48 KB stages: 193 KB of shared memory; 2 x 256 tensor-memory columns), CTAs of six warps:
//   warp 0 lane 0   TMA producer over the CTA's tiles and their K chunks (one running chunk count: the stage ring
//                   carries on from tile to tile)
//   warp 1 lane 0   MMA issuer: tile i accumulates in tensor memory columns (i & 1) x 256, after the epilogue has
//                   released that half (tempty); the tile's last commit signals the epilogue (tfull)
//   warps 2 - 5     epilogue: warp w reads accumulator lanes 32 (w mod 4) .. + 31 of tile i while the MMAs of tile
//                   i + 1 run in the other half, then releases the half (one arrival a warp)
// A CTA takes `tpc` consecutive tiles of the rasterised order and exits: short-lived enough that the LU's panel
// kernel (a cooperative launch on the other stream) still finds SMs, long enough that all but the last tile's
// epilogue run under MMAs. Every wait is bounded as in k_umma_update; on a time-out the CTA records
// M25_DEV_TIMEOUT, waits (bounded) for its loads and MMAs in flight, frees its tensor memory and returns.
constexpr int P_STAGES = 4;
constexpr int P_SMEM_BYTES = P_STAGES * STAGE_BYTES + 1024 + 256;
constexpr unsigned P_TMEM_COLS = 512;
static_assert(P_SMEM_BYTES <= 227 * 1024, "four stages in shared memory");

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void raster_tile(int pid, int nm, int nn, int &m0, int &n0)
{
    const int group = pid / (RASTER * nn), first = group * RASTER;
    const int rows = min(nm - first, RASTER);
    const int in_group = pid - group * RASTER * nn;
    m0 = (first + in_group % rows) * BM;
    n0 = (in_group / rows) * BN;
}

__global__ void __launch_bounds__(192, 1) k_umma_runs(float *C, long ldc_f, int Mp, int Nc, int kchunks, int tpc,
                                                       int nm, int nn,
                                                       const __grid_constant__ CUtensorMap mAhi,
                                                       const __grid_constant__ CUtensorMap mAlo,
                                                       const __grid_constant__ CUtensorMap mBhi,
                                                       const __grid_constant__ CUtensorMap mBlo, int *err)
{
    extern __shared__ unsigned char smem_raw[];
    const uint32_t base_raw = smem_u32(smem_raw);
    const uint32_t base = (base_raw + 1023) & ~1023u;
    const uint32_t bars = base + P_STAGES * STAGE_BYTES;
    // full[s] at bars + 8 s, empty[s] at bars + 32 + 8 s, tfull[a] at bars + 64 + 8 a, tempty[a] at bars + 80 + 8 a,
    // done at bars + 96, the tensor-memory address at bars + 104
    const uint32_t full0 = bars, empty0 = bars + 8 * P_STAGES, tfull0 = bars + 16 * P_STAGES,
                   tempty0 = tfull0 + 16, done = tempty0 + 16;
    volatile uint32_t *tmem_slot = reinterpret_cast<volatile uint32_t *>(smem_raw + (done + 8 - base_raw));
    __shared__ int abort_flag;
    __shared__ int issued_k, consumed_k;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = nm * nn;                                    // the tile grid: nm row tiles x nn column tiles
    const int t0 = blockIdx.x * tpc, t1 = min(ntiles, t0 + tpc);

    if (threadIdx.x == 0) {
        abort_flag = 0;
        for (int st = 0; st < P_STAGES; ++st) { mbar_init(full0 + 8 * st, 1); mbar_init(empty0 + 8 * st, 1); }
        for (int a = 0; a < 2; ++a) { mbar_init(tfull0 + 8 * a, 1); mbar_init(tempty0 + 8 * a, 4); }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issued_k = 0;
        consumed_k = 0;
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32((const void *)tmem_slot)), "r"(P_TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    volatile int *abort = &abort_flag;

    if (warp == 0 && lane == 0) {
        // producer
        int kg = 0;
        for (int t = t0; t < t1 && !*abort; ++t) {
            int m0, n0;
            raster_tile(t, nm, nn, m0, n0);
            for (int kc = 0; kc < kchunks; ++kc, ++kg) {
                const int st = kg % P_STAGES;
                if (kg >= P_STAGES && !mbar_wait(empty0 + 8 * st, ((kg / P_STAGES) - 1) & 1, abort)) break;
                const uint32_t sb = base + st * STAGE_BYTES;
                mbar_expect_tx(full0 + 8 * st, STAGE_BYTES);
                const int x = kc * BKF;
                tma_load_2d(sb, &mAhi, x, m0, full0 + 8 * st);
                tma_load_2d(sb + A_BYTES, &mAlo, x, m0, full0 + 8 * st);
                tma_load_2d(sb + 2 * A_BYTES, &mBhi, x, n0, full0 + 8 * st);
                tma_load_2d(sb + 2 * A_BYTES + B_BYTES, &mBlo, x, n0, full0 + 8 * st);
                issued_k = kg + 1;
            }
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        int kg = 0, i = 0;
        for (int t = t0; t < t1 && !*abort; ++t, ++i) {
            const int a = i & 1, use = i >> 1;
            if (use > 0 && !mbar_wait(tempty0 + 8 * a, (use - 1) & 1, abort)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t d = tmem + (uint32_t)(a * 256);
            bool ok = true;
            for (int kc = 0; kc < kchunks; ++kc, ++kg) {
                const int st = kg % P_STAGES;
                if (!mbar_wait(full0 + 8 * st, (kg / P_STAGES) & 1, abort)) { ok = false; break; }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t sb = base + st * STAGE_BYTES;
                const uint32_t aH = sb, aL = sb + A_BYTES, bH = sb + 2 * A_BYTES, bL = sb + 2 * A_BYTES + B_BYTES;
#pragma unroll
                for (int k = 0; k < BKF / 8; ++k) {
                    const uint32_t off = k * 32;
                    umma_tf32(d, sdesc(aL + off), sdesc(bH + off), (kc > 0 || k > 0) ? 1u : 0u);
                    umma_tf32(d, sdesc(aH + off), sdesc(bL + off), 1u);
                    umma_tf32(d, sdesc(aH + off), sdesc(bH + off), 1u);
                }
                umma_commit(empty0 + 8 * st);
                consumed_k = kg + 1;
            }
            if (!ok) break;
            umma_commit(tfull0 + 8 * a);                     // the tile's accumulator is complete
        }
        umma_commit(done);                                   // (every MMA issued so far complete)
    } else if (warp >= 2) {
        // epilogue: warp w reads tensor-memory lanes 32 (w mod 4) .. + 31
        const int q = warp & 3;
        int i = 0;
        for (int t = t0; t < t1; ++t, ++i) {
            const int a = i & 1, use = i >> 1;
            const bool ok = mbar_wait(tfull0 + 8 * a, use & 1, abort);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (!__all_sync(0xffffffffu, ok && !*abort)) break;          // warp-uniform: tcgen05.ld is .sync.aligned
            int m0, n0;
            raster_tile(t, nm, nn, m0, n0);
            const int row = m0 + q * 32 + lane;
            for (int c0 = 0; c0 < BN; c0 += 32) {
                uint32_t v[32];
                const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(a * 256 + c0);
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
                             "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                             : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
                               "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
                               "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
                               "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]),
                               "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                             : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (row < Mp) {
                    float cv[32];
                    float *pc = C + (size_t)(n0 + c0) * ldc_f + row;
                    const int nv = min(32, Nc - (n0 + c0));
#pragma unroll
                    for (int j = 0; j < 32; ++j) cv[j] = j < nv ? __ldcs(pc + (size_t)j * ldc_f) : 0.f;
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        if (j < nv) __stcs(pc + (size_t)j * ldc_f, cv[j] - __uint_as_float(v[j]));
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(tempty0 + 8 * a);     // this half may take the next tile's accumulation
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile int never = 0;
        if (*abort) {
            dev_error(err, M25_DEV_TIMEOUT);
            // loads still in flight would land in this CTA's shared memory after it exits: wait for them (bounded)
            for (int kc = consumed_k; kc < issued_k; ++kc)
                mbar_wait(full0 + 8 * (kc % P_STAGES), (kc / P_STAGES) & 1, &never);
        }
        never = 0;
        mbar_wait(done, 0, &never);                          // the MMAs issued (they read shared, write tensor memory)
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(P_TMEM_COLS) : "memory");
}

// A' (2M x Kp floats, row-major, hi and lo) from L (M x K complex, column-major, lda): rows 2m / 2m+1 hold
// [Lr, -Li] / [Li, Lr] for every k; columns 2K .. Kp zero. A 32 x 32 (m, k) tile through shared memory so both the
// read (along m) and the write (along k) are coalesced.
__global__ void k_split_A(const float *L, long lda, int M, int K, int Kp, float *Ahi, float *Alo)
{
    __shared__ float2 t[32][33];
    const int mb = blockIdx.y * 32, kb = blockIdx.x * 32;
    for (int i = threadIdx.y; i < 32; i += 8) {              // i: k within the tile, threadIdx.x: m
        int m = mb + threadIdx.x, k = kb + i;
        float2 z = make_float2(0.f, 0.f);
        if (m < M && k < K) z = reinterpret_cast<const float2 *>(L)[(size_t)k * lda + m];
        t[i][threadIdx.x] = z;
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += 8) {              // i: m within the tile, threadIdx.x: k
        int m = mb + i, k = kb + threadIdx.x;
        if (m >= M || 2 * k >= Kp) continue;
        float2 z = t[threadIdx.x][i];
        float r0a = z.x, r0b = -z.y, r1a = z.y, r1b = z.x;
        float h;
        size_t o0 = (size_t)(2 * m) * Kp + 2 * k, o1 = o0 + Kp;
        h = tf32_rna(r0a); Ahi[o0] = h; Alo[o0] = tf32_rna(r0a - h);
        h = tf32_rna(r0b); Ahi[o0 + 1] = h; Alo[o0 + 1] = tf32_rna(r0b - h);
        h = tf32_rna(r1a); Ahi[o1] = h; Alo[o1] = tf32_rna(r1a - h);
        h = tf32_rna(r1b); Ahi[o1 + 1] = h; Alo[o1 + 1] = tf32_rna(r1b - h);
    }
}

// B' (N x Kp floats, row-major = U's columns as real, hi and lo), columns 2K .. Kp zero
__global__ void k_split_B(const float *U, long lda, int K, int N, int Kp, float *Bhi, float *Blo)
{
    long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= (long)N * Kp) return;
    int n = e / Kp, j = e % Kp;
    float x = j < 2 * K ? U[(size_t)n * 2 * lda + j] : 0.f;
    float h = tf32_rna(x);
    Bhi[e] = h; Blo[e] = tf32_rna(x - h);
}

typedef CUresult (*EncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn()
{
    static EncodeTiled fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiled)p;
    }
    return fn;
}

// a row-major rows x cols (floats, row pitch pitch_f) matrix, box of BKF floats x box_rows rows, swizzled rows
int make_map(CUtensorMap *m, const float *ptr, long rows, long cols, long pitch_f, int box_rows)
{
    EncodeTiled enc = encode_fn();
    if (!enc) { m25_set_error("cuTensorMapEncodeTiled is not available"); return M25_ECUDA; }
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)pitch_f * 4};
    cuuint32_t box[2] = {(cuuint32_t)BKF, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)ptr, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE,
                     SWZ_BYTES == 128 ? CU_TENSOR_MAP_SWIZZLE_128B :
                     SWZ_BYTES == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) { m25_set_error("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")"); return M25_ECUDA; }
    return M25_OK;
}

}  // namespace

// Tiles a CTA of the tensor-core update: 1 runs k_umma_update (one tile a CTA, two CTAs an SM), more runs k_umma_runs
// with that many consecutive tiles a CTA, for updates of at least `min_tiles` tiles (default two an SM; smaller ones
// keep one tile a CTA). M25_UMMA_TPC in the environment overrides the count.
static int g_umma_tpc = 1, g_umma_min = -1;

extern "C" int m25_set_umma_tiles(int tiles, int min_tiles)
{
    M25_REQUIRE(tiles >= 1 && tiles <= 64, "m25_set_umma_tiles: 1 to 64 tiles a CTA");
    g_umma_tpc = tiles;
    g_umma_min = min_tiles;
    return M25_OK;
}

static int umma_tiles_per_cta(int ntiles)
{
    int t = g_umma_tpc;
    if (const char *e = getenv("M25_UMMA_TPC")) t = std::max(1, std::min(64, atoi(e)));
    int sms = 148, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int need = g_umma_min >= 0 ? g_umma_min : 2 * sms;
    return (t > 1 && ntiles >= need) ? t : 1;
}

size_t m25_umma_workspace(int n, int nb)
{
    (void)nb;
    const size_t Kp = 512;                                   // 2 x the outer panel (256), a multiple of BKF
    return (2 * (size_t)(2 * n) * Kp + 2 * (size_t)n * Kp) * sizeof(float) + 4096;
}

// C (M x Nc complex, column-major, lda) -= L (M x K) U (K x Nc), both inside the same column-major matrix
int m25_umma_trailing(float *C, long lda, int M, int Nc, int K, const float *L21, const float *U12, void *work,
                      size_t work_bytes, cudaStream_t s)
{
    M25_REQUIRE(K >= 1 && K <= 256, "m25_umma_trailing: depth 1 to 256");
    if (M <= 0 || Nc <= 0) return M25_OK;
    const int Kp = (2 * K + BKF - 1) / BKF * BKF;
    const size_t need = (2 * (size_t)(2 * M) * Kp + 2 * (size_t)Nc * Kp) * sizeof(float);
    M25_REQUIRE(need <= work_bytes, "m25_umma_trailing: workspace too small");
    float *Ahi = (float *)work, *Alo = Ahi + (size_t)(2 * M) * Kp;
    float *Bhi = Alo + (size_t)(2 * M) * Kp, *Blo = Bhi + (size_t)Nc * Kp;
    dim3 ga((Kp / 2 + 31) / 32, (M + 31) / 32), ba(32, 8);
    k_split_A<<<ga, ba, 0, s>>>(L21, lda, M, K, Kp, Ahi, Alo);
    M25_LAUNCH_CHECK("k_split_A");
    long tb = (long)Nc * Kp;
    k_split_B<<<(tb + 255) / 256, 256, 0, s>>>(U12, lda, K, Nc, Kp, Bhi, Blo);
    M25_LAUNCH_CHECK("k_split_B");
    CUtensorMap mAhi, mAlo, mBhi, mBlo;
    int rc;
    if ((rc = make_map(&mAhi, Ahi, 2L * M, Kp, Kp, BM))) return rc;
    if ((rc = make_map(&mAlo, Alo, 2L * M, Kp, Kp, BM))) return rc;
    if ((rc = make_map(&mBhi, Bhi, Nc, Kp, Kp, BN))) return rc;
    if ((rc = make_map(&mBlo, Blo, Nc, Kp, Kp, BN))) return rc;
    const int nm = (2 * M + BM - 1) / BM, nn = (Nc + BN - 1) / BN, ntiles = nm * nn;
    const int tpc = umma_tiles_per_cta(ntiles);
    if (tpc <= 1) {                                          // one tile a CTA, two CTAs an SM
        static bool attr = false;
        if (!attr) {
            M25_CHECK(cudaFuncSetAttribute(k_umma_update, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES));
            attr = true;
        }
        dim3 grid(nn, nm);
        k_umma_update<<<grid, 128, SMEM_BYTES, s>>>(C, 2 * lda, 2 * M, Nc, Kp / BKF, mAhi, mAlo, mBhi, mBlo,
                                                    m25_dev_err_word());
        M25_LAUNCH_CHECK("k_umma_update");
        return M25_OK;
    }
    static bool pattr = false;
    if (!pattr) {
        M25_CHECK(cudaFuncSetAttribute(k_umma_runs, cudaFuncAttributeMaxDynamicSharedMemorySize, P_SMEM_BYTES));
        pattr = true;
    }
    k_umma_runs<<<(ntiles + tpc - 1) / tpc, 192, P_SMEM_BYTES, s>>>(C, 2 * lda, 2 * M, Nc, Kp / BKF, tpc, nm, nn, mAhi,
                                                                     mAlo, mBhi, mBlo, m25_dev_err_word());
    M25_LAUNCH_CHECK("k_umma_runs");
    return M25_OK;
}

extern "C" int m25_umma_available(void) { return 1; }

// C (M x N complex64, column-major, ldc) -= L (M x K) U (K x N), column-major with leading dimension ld each, on
// the tensor cores (3xTF32). The LU's trailing update as a call of its own (C, L, U in one matrix there).
extern "C" int m25_cgemm_update_tf32(float *d_C, long ld, int M, int N, int K, const float *d_L, const float *d_U,
                                     void *d_work, size_t work_bytes, void *stream)
{
    return m25_umma_trailing(d_C, ld, M, N, K, d_L, d_U, d_work, work_bytes, (cudaStream_t)stream);
}
