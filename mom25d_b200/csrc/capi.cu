// capi.cu - the C ABI's common entry points: version, errors (a thread-local message; a device error word that
// kernels set instead of trapping), device information.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "common.cuh"

#include <atomic>

static thread_local std::string g_err;
static std::atomic<long long> g_launches{0};

void m25_note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

// The number of kernels this library has launched since it was loaded (every launch site counts itself).
extern "C" long long m25_launch_count(void) { return g_launches.load(); }

void m25_set_error(const std::string &msg) { g_err = msg; }

int m25_cuda_status(cudaError_t e, const char *where)
{
    g_err = std::string(where) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return M25_ECUDA;
}

// one device error word per device, allocated on first use
static int *g_dev_err[64];
static std::mutex g_mu;

int *m25_noalloc_status_word();

int *m25_dev_err_word()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_dev_err[dev]) {
        int *p = nullptr;
        if (cudaMalloc(&p, sizeof(int)) != cudaSuccess) return nullptr;
        cudaMemset(p, 0, sizeof(int));
        cudaDeviceSynchronize();
        g_dev_err[dev] = p;
    }
    return g_dev_err[dev];
}

extern "C" const char *m25_version(void) { return "mom25d_b200 0.1 (sm_100a)"; }

extern "C" const char *m25_last_error(void) { return g_err.c_str(); }

extern "C" int m25_device_info(int *sm_count, size_t *free_bytes, size_t *total_bytes)
{
    int dev = 0;
    M25_CHECK(cudaGetDevice(&dev));
    if (sm_count) M25_CHECK(cudaDeviceGetAttribute(sm_count, cudaDevAttrMultiProcessorCount, dev));
    size_t f = 0, t = 0;
    M25_CHECK(cudaMemGetInfo(&f, &t));
    if (free_bytes) *free_bytes = f;
    if (total_bytes) *total_bytes = t;
    return M25_OK;
}

// Synchronises the stream and reads (then clears) the device error words: M25_EDEVICE with the code if a kernel
// reported one (an index out of range, a bounded wait that gave up, a zero pivot). Two words per device: the
// library's, and m25_getrs_noalloc's own where that has run. Both are read and both are cleared, so that a code
// left in one cannot make a later call fail; the first nonzero code is the one reported.
extern "C" int m25_sync_check(void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    M25_CHECK(cudaStreamSynchronize(s));
    int *w = m25_dev_err_word();
    if (!w) { g_err = "m25_sync_check: no device error word"; return M25_ECUDA; }
    int code = 0, code2 = 0;
    M25_CHECK(cudaMemcpy(&code, w, sizeof(int), cudaMemcpyDeviceToHost));
    int *nw = m25_noalloc_status_word();               // m25_getrs_noalloc's own word, where it has run
    if (nw) {
        M25_CHECK(cudaMemcpy(&code2, nw, sizeof(int), cudaMemcpyDeviceToHost));
        if (code2) M25_CHECK(cudaMemset(nw, 0, sizeof(int)));
    }
    if (!code) code = code2;
    if (code) {
        M25_CHECK(cudaMemset(w, 0, sizeof(int)));
        char buf[128];
        snprintf(buf, sizeof buf, "a kernel reported device code %d (%s)", code,
                 code == M25_DEV_TIMEOUT ? "a bounded wait gave up" : code == M25_DEV_INDEX ? "index out of range" :
                 code == M25_DEV_ZEROPIV ? "zero pivot: singular factor" : "unknown");
        g_err = buf;
        return M25_EDEVICE;
    }
    return M25_OK;
}

// ---- failure detection without a fault: a bounded wait that runs out ------------------------------------------------
// The grid barrier of the cooperative kernels (grid_sync), entered by one block that waits for a second block which
// is never launched: the wait ends at its iteration limit, the device error word gets M25_DEV_TIMEOUT and the
// kernel returns. m25_sync_check then reports M25_EDEVICE and the context stays usable.
static __device__ unsigned g_selftest_barrier[2];

__global__ void k_wait_selftest(int *err)
{
    if (threadIdx.x == 0) { g_selftest_barrier[0] = 0u; g_selftest_barrier[1] = 0u; }
    GridBarrier b{&g_selftest_barrier[0], &g_selftest_barrier[1]};
    unsigned phase = 0;
    grid_sync(b, 2u, phase, err);
}

extern "C" int m25_wait_selftest(void *stream)
{
    int *err = m25_dev_err_word();
    if (!err) { g_err = "m25_wait_selftest: no device error word"; return M25_ECUDA; }
    k_wait_selftest<<<1, 32, 0, (cudaStream_t)stream>>>(err);
    M25_LAUNCH_CHECK("k_wait_selftest");
    return M25_OK;
}
