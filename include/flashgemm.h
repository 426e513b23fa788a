/* flashgemm chain API, B200 implementation.
 *
 * Drop-in for the reference's multigemm interface, declared at
 * multigemm/src/flashgemm.h:17-25 (implemented there in multigemm/src/flashgemm.c).
 * Same names, same argument meaning, same variadic ABI: after num_gemm come
 * num_gemm triples (T *A_i, long M_i, long K_i), read as (pointer, long, long)
 * exactly as flashgemm.c:56-60 reads them, so callers must pass long.
 *
 * Shapes (reference orientation, all row-major, host memory):
 *   B   : K_1 x N
 *   A_i : M_i x K_i, with K_{i+1} = M_i
 *   C   : M_n x N,   C = A_n * (... * (A_2 * (A_1 * B)))
 *
 * The computation runs on the current CUDA device (sm_100a); the call copies
 * the operands in, runs the chain, copies C out and returns, like the
 * reference's blocking call. Results follow the reference's own semantics by
 * default (see flashgemm_b200.h: fg_set_semantics), including its BF16/INT8
 * between-stage panel permutation and INT8 tail-row behaviour.
 *
 * Errors: like the reference, these return nothing. Where the reference prints
 * and returns (K % 2 != 0, flashgemm.c:13-22), this prints the same message
 * and returns without touching C; every failure also sets fg_last_error(). */
#ifndef FLASHGEMM_B200_FLASHGEMM_H
#define FLASHGEMM_B200_FLASHGEMM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Thread count the reference's OpenMP team uses (flashgemm.c:6). Here it is
 * stored and read back, and changes no result: the GPU uses no host threads,
 * and the reference's 32-column panels always start at multiples of 32
 * columns, which is where the reference's strips put them whenever its strip
 * width 16 * ceil(ceil(N / 16) / T) is a multiple of 32 (flashgemm.c:40-52),
 * i.e. on every input whose result the reference defines. Replaces
 * flashgemm.h:17. */
extern int flashgemm_thread_num;

/* Replaces flashgemm.h:19 / flashgemm.c:8-11. */
void flashgemm_set_thread_num(int num);

/* FP32 chain. Replaces flashgemm.h:21 / flashgemm.c:24-156. */
void flashgemm_multi_f32f32f32(float *C, float *B, long N, int num_gemm, ...);

/* BF16 inputs (raw bits in uint16_t), FP32 accumulation, FP32 C.
 * Replaces flashgemm.h:23 / flashgemm.c:158-290. */
void flashgemm_multi_bf16bf16f32(float *C, uint16_t *B, long N, int num_gemm, ...);

/* INT8 chain, int32 C. As in the reference's kernels (kernel_int8.h:56), the
 * bytes of A_i (declared int8_t) are multiplied as UNSIGNED values and the
 * bytes of B (declared uint8_t) as SIGNED values.
 * Replaces flashgemm.h:25 / flashgemm.c:292-424. */
void flashgemm_multi_int8uint8int32(int *C, uint8_t *B, long N, int num_gemm, ...);

#ifdef __cplusplus
}
#endif

#endif
