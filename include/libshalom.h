/* singlegemm (LibShalom) FP32 SGEMM API, B200 implementation.
 *
 * C = A * B, row-major, A: M x K, B: K x N, C: M x N, host memory; no alpha or
 * beta, C fully overwritten. Results are bit-identical to the reference's
 * (one FP32 FMA per k in increasing k, K cut into blocks of 2048 whose partial
 * sums are added into C, singlegemm/src/NN_mp.h:13) with the default plain
 * FP32 kernel; fg_set_f32_algo(FG_F32_3XTF32) selects split-precision 3xTF32
 * on the tensor cores instead.
 *
 * The reference defines these with C++ linkage; the library exports both the
 * C names declared here and the C++ (mangled) names, so objects compiled
 * against either the reference's headers or this one link. */
#ifndef FLASHGEMM_B200_LIBSHALOM_H
#define FLASHGEMM_B200_LIBSHALOM_H

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces singlegemm/FP32_ID23.c:35-62. transb == 0 (NN) computes C = A * B;
 * transb == 1 (NT) does nothing, as in the reference, which only picks a
 * thread grid there (:39-43). transa is ignored, as in the reference. */
void LibShalom_sgemm_mp(int transa, int transb, float *C, float *A, float *B, long M, long N,
                        long K);

/* Replaces singlegemm/src/set_TmTn.h:61. Accepted and recorded; the GPU has no
 * host thread grid. */
void LibShalom_set_thread_nums(int num);

/* Replace singlegemm/src/NN_mp.h:11 and :245. NUM, Tm and Tn are accepted and
 * ignored; both compute C = A * B. */
void Small_NGM_NN_SGEMM(float *C, float *A, float *B, long M, long N, long K, int NUM, int Tm,
                        int Tn);
void Small_MGN_NN_SGEMM(float *C, float *A, float *B, long M, long N, long K, int NUM, int Tm,
                        int Tn);

#ifdef __cplusplus
}
#endif

#endif
