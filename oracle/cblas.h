/* Test infrastructure only: the oracle.
 *
 * Stand-in for OpenBLAS's cblas.h, which the reference's singlegemm benchmark
 * (singlegemm/FP32_ID23.c:6,67,125) includes for its correctness check. The
 * benchmark's main() is renamed away in ref_singlegemm_shim.cpp, so these are
 * only here to let that file compile; the naive loop is never timed. */
#ifndef FG_ORACLE_CBLAS_STUB_H
#define FG_ORACLE_CBLAS_STUB_H
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112 };
static inline void openblas_set_num_threads(int) {}
static inline void cblas_sgemm(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, long M, long N,
                               long K, float alpha, const float *A, long lda, const float *B,
                               long ldb, float beta, float *C, long ldc)
{
    for (long i = 0; i < M; ++i)
        for (long j = 0; j < N; ++j) {
            float s = 0.f;
            for (long k = 0; k < K; ++k) s += A[i * lda + k] * B[k * ldb + j];
            C[i * ldc + j] = alpha * s + beta * C[i * ldc + j];
        }
}
#endif
