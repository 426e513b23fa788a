/* Test infrastructure only: the oracle. Nothing in the product links this.
 *
 * A CPU restatement, in plain C, of the arithmetic of the reference's hot path
 * (AnonymousJune/flashgemm): the FP32 single GEMM and the FP32 / BF16 / INT8
 * GEMM chains C = A_n*(...*(A_1*B)), in the reference's orientation:
 *   B   : K1 x N   row-major (the activation panel source)
 *   A_i : M_i x K_i row-major, K_{i+1} = M_i
 *   C   : M_n x N  row-major
 *
 * Two semantics: FG_ORC_REF reproduces what the compiled reference computes
 * (including its inter-stage panel permutation and INT8 tail behaviour);
 * FG_ORC_MATH is the mathematical chain with the same narrowing points. */
#ifndef FG_ORACLE_H
#define FG_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { FG_ORC_REF = 0, FG_ORC_MATH = 1 };

uint16_t orc_f32_to_bf16_rne(float x);
uint16_t orc_f32_to_bf16_trunc(float x);
float orc_bf16_to_f32(uint16_t h);
int8_t orc_sat_s8(int32_t v);

void orc_sgemm_f64(const float *A, const float *B, double *C, long M, long N, long K);
void orc_sgemm_f32(const float *A, const float *B, float *C, long M, long N, long K,
                   long kblock);

void orc_chain_f32(float *C, const float *B, long N, int n, const float *const *A,
                   const long *M, const long *K);
void orc_chain_f64(double *C, const float *B, long N, int n, const float *const *A,
                   const long *M, const long *K);

int orc_chain_bf16(float *C, const uint16_t *B, long N, int n, const uint16_t *const *A,
                   const long *M, const long *K, int mode, int threads);
int orc_chain_int8(int32_t *C, const uint8_t *B, long N, int n, const int8_t *const *A,
                   const long *M, const long *K, int mode, int threads);

long orc_strip_width(long N, int threads);
double orc_rel_frob(const float *x, const double *ref, long count);

#ifdef __cplusplus
}
#endif
#endif
