// umma.cu - the complex64 LU's trailing update on the tensor cores (tcgen05, 3xTF32). Placeholder until the
// tensor-core kernel lands: asking for it is an error, never a silent fallback.
#include "common.cuh"

size_t m25_umma_workspace(int n, int nb) { (void)n; (void)nb; return 0; }

int m25_umma_trailing(float *A, long lda, int M, int Ncol, int K, const float *L21, const float *U12, void *work,
                      size_t work_bytes, cudaStream_t s)
{
    (void)A; (void)lda; (void)M; (void)Ncol; (void)K; (void)L21; (void)U12; (void)work; (void)work_bytes; (void)s;
    m25_set_error("m25_getrf: the tensor-core (3xTF32) trailing update is not built in this library");
    return M25_EINVAL;
}
