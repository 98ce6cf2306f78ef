// noalloc.cu - m25_getrs_noalloc: the triangular solves of m25_getrs on file-scope device scratch instead of memory
// taken from the stream-ordered allocator at each call. Its own compilation unit, so that the scratch (a module
// global) is set up only in processes that use this entry point.
#include <mutex>

#include "common.cuh"

// The scratch of m25_getrs_noalloc: the diagonal-block inverses, the permutation, two n x nrhs work vectors and
// the solves' flags (the layout of the 64-row-block solves, m25_getrs_aux_bytes_basic; this entry point
// always solves that way). Its contents need not start at zero: every call zeroes the
// flags it waits on before its solves read them.
static __device__ __align__(256) unsigned char g_getrs_scratch[M25_GETRS_NOALLOC_MAX_BYTES];
// The device status word of those solves (zero at module load; a bounded wait that gave up writes its code here).
static __device__ int g_getrs_status;

int m25_getrs_on_scratch(const void *d_LU, long lda, int n, const int *d_ipiv, int single, void *d_aux,
                         size_t aux_bytes, int *d_err, void *d_B, int nrhs, cudaStream_t s);
size_t m25_getrs_aux_bytes_basic(int n, int single);

namespace {
struct Scratch { void *aux = nullptr; int *status = nullptr; };
Scratch g_dev[64];
std::mutex g_mu;

// The symbols' device addresses on the current device, looked up once per device (with that device current).
int scratch_of_current_device(Scratch *out)
{
    int dev = -1;
    M25_CHECK(cudaGetDevice(&dev));
    M25_REQUIRE(dev >= 0 && dev < 64, "m25_getrs_noalloc: device index above 63");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_dev[dev].aux) {
        void *aux = nullptr, *st = nullptr;
        M25_CHECK(cudaGetSymbolAddress(&aux, g_getrs_scratch));
        M25_CHECK(cudaGetSymbolAddress(&st, g_getrs_status));
        g_dev[dev].aux = aux;
        g_dev[dev].status = (int *)st;
    }
    *out = g_dev[dev];
    return M25_OK;
}
}  // namespace

// The status word of the current device, or null where m25_getrs_noalloc has not run on it (m25_sync_check).
int *m25_noalloc_status_word()
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    return g_dev[dev].status;
}

extern "C" int m25_getrs_noalloc(const void *d_LU, long lda, int n, const int *d_ipiv, int single, void *d_B,
                                 int nrhs, void *stream)
{
    M25_REQUIRE(d_LU && d_ipiv && d_B && n >= 1 && lda >= n, "m25_getrs_noalloc: LU, ipiv, B, n >= 1");
    M25_REQUIRE(nrhs >= 1 && nrhs <= 16, "m25_getrs_noalloc: 1 to 16 right-hand sides a call");
    const size_t need = m25_getrs_aux_bytes_basic(n, single);     // the 64-row-block solves' data
    if (need > (size_t)M25_GETRS_NOALLOC_MAX_BYTES) {
        char buf[200];
        snprintf(buf, sizeof buf, "m25_getrs_noalloc: n = %d (%s) needs %zu scratch bytes, above the fixed %zu "
                 "(use m25_getrs, or m25_getrs_prepare / m25_getrs_aux with your own buffer)", n,
                 single ? "complex64" : "complex128", need, (size_t)M25_GETRS_NOALLOC_MAX_BYTES);
        m25_set_error(buf);
        return M25_EINVAL;
    }
    Scratch sc;
    int rc = scratch_of_current_device(&sc);
    if (rc) return rc;
    return m25_getrs_on_scratch(d_LU, lda, n, d_ipiv, single, sc.aux, (size_t)M25_GETRS_NOALLOC_MAX_BYTES, sc.status,
                                d_B, nrhs, (cudaStream_t)stream);
}
