// common.cuh - shared device helpers of libmom25d_b200: complex arithmetic on interleaved (re, im) pairs, the
// packed mesh / table views the kernels read, a bounded grid barrier, and the error plumbing of the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "../../include/mom25d_b200.h"

// ---- complex arithmetic (interleaved re, im: the layout of numpy complex128 / complex64) ----------------------------
template <typename R> struct cpx { R x, y; };
template <typename R> struct vec2_of;
template <> struct vec2_of<double> { typedef double2 type; };
template <> struct vec2_of<float> { typedef float2 type; };

template <typename R> __host__ __device__ __forceinline__ cpx<R> mk(R a, R b) { cpx<R> c; c.x = a; c.y = b; return c; }
template <typename R> __host__ __device__ __forceinline__ cpx<R> operator+(cpx<R> a, cpx<R> b) { return mk(a.x + b.x, a.y + b.y); }
template <typename R> __host__ __device__ __forceinline__ cpx<R> operator-(cpx<R> a, cpx<R> b) { return mk(a.x - b.x, a.y - b.y); }
template <typename R> __host__ __device__ __forceinline__ cpx<R> operator*(cpx<R> a, cpx<R> b) { return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename R> __host__ __device__ __forceinline__ cpx<R> operator*(cpx<R> a, R s) { return mk(a.x * s, a.y * s); }
template <typename R> __host__ __device__ __forceinline__ cpx<R> operator*(R s, cpx<R> a) { return mk(a.x * s, a.y * s); }
template <typename R> __host__ __device__ __forceinline__ cpx<R> operator/(cpx<R> a, R s) { return mk(a.x / s, a.y / s); }
template <typename R> __host__ __device__ __forceinline__ cpx<R> &operator+=(cpx<R> &a, cpx<R> b) { a.x += b.x; a.y += b.y; return a; }
template <typename R> __host__ __device__ __forceinline__ cpx<R> &operator-=(cpx<R> &a, cpx<R> b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename R> __host__ __device__ __forceinline__ cpx<R> conj(cpx<R> a) { return mk(a.x, -a.y); }
template <typename R> __host__ __device__ __forceinline__ R abs1(cpx<R> a) { return fabs(a.x) + fabs(a.y); }
// a / b by Smith's method (the scaled quotient; no overflow for large |b|)
template <typename R> __host__ __device__ __forceinline__ cpx<R> cdiv(cpx<R> a, cpx<R> b)
{
    if (fabs(b.x) >= fabs(b.y)) {
        R r = b.y / b.x, d = b.x + b.y * r;
        return mk((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    }
    R r = b.x / b.y, d = b.x * r + b.y;
    return mk((a.x * r + a.y) / d, (a.y * r - a.x) / d);
}
// a += b * c
template <typename R> __host__ __device__ __forceinline__ void cfma(cpx<R> &a, cpx<R> b, cpx<R> c)
{
    a.x = fma(b.x, c.x, a.x); a.x = fma(-b.y, c.y, a.x);
    a.y = fma(b.x, c.y, a.y); a.y = fma(b.y, c.x, a.y);
}
// a -= b * c
template <typename R> __host__ __device__ __forceinline__ void cfms(cpx<R> &a, cpx<R> b, cpx<R> c)
{
    a.x = fma(-b.x, c.x, a.x); a.x = fma(b.y, c.y, a.x);
    a.y = fma(-b.x, c.y, a.y); a.y = fma(-b.y, c.x, a.y);
}

typedef cpx<double> zd;
typedef cpx<float> zf;

template <typename R> __device__ __forceinline__ cpx<R> ldc(const R *p, size_t i)
{
    typedef typename vec2_of<R>::type V;
    V v = reinterpret_cast<const V *>(p)[i];
    return mk(v.x, v.y);
}
template <typename R> __device__ __forceinline__ void stc(R *p, size_t i, cpx<R> c)
{
    typedef typename vec2_of<R>::type V;
    V v; v.x = c.x; v.y = c.y;
    reinterpret_cast<V *>(p)[i] = v;
}

// ---- FP64 tensor-core product (mma.sync; tcgen05 has no FP64 kind) ------------------------------------------------
// D (16 x 8) += A (16 x 8, row) B (8 x 8, col), FP64. Lane l = 4 g + t holds A[g][t], A[g + 8][t], A[g][t + 4],
// A[g + 8][t + 4]; B[t][g], B[t + 4][g]; D[g][2 t], D[g][2 t + 1], D[g + 8][2 t], D[g + 8][2 t + 1].
__device__ __forceinline__ void dmma_16x8x8(double (&d)[4], const double (&a)[4], const double (&b)[2])
{
    asm("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// ---- error plumbing ---------------------------------------------------------------------------------------------------
void m25_set_error(const std::string &msg);
int m25_cuda_status(cudaError_t e, const char *where);
void m25_note_launch();          // counts this library's kernel launches (m25_launch_count)
#define M25_CHECK(call)                                                                                    \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return m25_cuda_status(e_, #call);                                          \
    } while (0)
#define M25_LAUNCH_CHECK(what)                                                                             \
    do {                                                                                                   \
        m25_note_launch();                                                                                 \
        cudaError_t e_ = cudaGetLastError();                                                               \
        if (e_ != cudaSuccess) return m25_cuda_status(e_, what);                                           \
    } while (0)
#define M25_REQUIRE(cond, msg)                                                                             \
    do {                                                                                                   \
        if (!(cond)) { m25_set_error(msg); return M25_EINVAL; }                                            \
    } while (0)

// device-side error word: kernels that detect a bad index or a barrier that gave up write a code here (never trap)
__device__ __forceinline__ void dev_error(int *err, int code)
{
    if (err) atomicCAS(err, 0, code);
}

// ---- a bounded grid barrier for cooperative (co-resident) launches -------------------------------------------------
// count / gen live in global memory (zeroed before the launch). Every block arrives once per phase; the last one
// bumps the generation. A wait that exceeds `limit` polls records M25_DEV_TIMEOUT in *err and returns false, so a
// stuck phase ends the kernel instead of hanging the GPU.
struct GridBarrier {
    unsigned *count;
    unsigned *gen;
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool grid_sync(GridBarrier b, unsigned nblocks, unsigned &phase, int *err)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        __threadfence();                                  // release: the CTA's writes (ordered by the barrier above)
        unsigned target = phase + 1;
        if (atomicAdd(b.count, 1u) == nblocks * target - 1) {
            __threadfence();                              // the last arrival: everyone's writes, then the release
            atomicExch(b.gen, target);
        } else {
            long it = 0;                                  // acquire spin; the limit and the error word every 1024
            while (ld_acquire_u32(b.gen) < target) {
                if ((++it & 1023) == 0) {
                    if (it > (1L << 22)) { ok = 0; dev_error(err, M25_DEV_TIMEOUT); break; }
                    if (err && *(volatile int *)err) { ok = 0; break; }
                }
            }
        }
    }
    __syncthreads();
    phase += 1;
    return ok;
}
