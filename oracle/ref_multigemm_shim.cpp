// Test infrastructure only: the oracle. Nothing in the product links this file.
//
// Builds the reference's own multigemm implementation from its sources where
// they lie (multigemm/src/flashgemm.c, which #includes the packing routines and
// the AVX-512 micro-kernels), with the public symbols renamed ref_* so that the
// reference and the B200 library can be loaded into one process, and adds
// fixed-arity wrappers that ctypes can call without variadic promotion rules.
//
// Reference interface: multigemm/src/flashgemm.h:17-25.

// The reference test mains include these before flashgemm.c (test_int8_3.c:1-5).
#include <stdio.h>
#include <stdlib.h>
#include <stdint.h>
#include <string.h>

#define flashgemm_thread_num ref_flashgemm_thread_num
#define flashgemm_set_thread_num ref_flashgemm_set_thread_num
#define flashgemm_multi_f32f32f32 ref_flashgemm_multi_f32f32f32
#define flashgemm_multi_bf16bf16f32 ref_flashgemm_multi_bf16bf16f32
#define flashgemm_multi_int8uint8int32 ref_flashgemm_multi_int8uint8int32
#include "multigemm/src/flashgemm.c"

#define T1(i) A[i], M[i], K[i]
#define CHAIN_SWITCH(fn, C, B, N, n)                                                       \
    switch (n) {                                                                           \
    case 1: fn(C, B, N, 1, T1(0)); break;                                                  \
    case 2: fn(C, B, N, 2, T1(0), T1(1)); break;                                           \
    case 3: fn(C, B, N, 3, T1(0), T1(1), T1(2)); break;                                    \
    case 4: fn(C, B, N, 4, T1(0), T1(1), T1(2), T1(3)); break;                             \
    case 5: fn(C, B, N, 5, T1(0), T1(1), T1(2), T1(3), T1(4)); break;                      \
    case 6: fn(C, B, N, 6, T1(0), T1(1), T1(2), T1(3), T1(4), T1(5)); break;               \
    case 7: fn(C, B, N, 7, T1(0), T1(1), T1(2), T1(3), T1(4), T1(5), T1(6)); break;        \
    case 8: fn(C, B, N, 8, T1(0), T1(1), T1(2), T1(3), T1(4), T1(5), T1(6), T1(7)); break; \
    default: return -1;                                                                    \
    }                                                                                      \
    return 0;

extern "C" {

void ref_set_threads(int t) { ref_flashgemm_set_thread_num(t); }
int ref_get_threads(void) { return ref_flashgemm_thread_num; }

int ref_chain_f32(float *C, float *B, long N, int n, float *const *A, const long *M,
                  const long *K)
{
    CHAIN_SWITCH(ref_flashgemm_multi_f32f32f32, C, B, N, n)
}

int ref_chain_bf16(float *C, uint16_t *B, long N, int n, uint16_t *const *A, const long *M,
                   const long *K)
{
    CHAIN_SWITCH(ref_flashgemm_multi_bf16bf16f32, C, B, N, n)
}

int ref_chain_int8(int *C, uint8_t *B, long N, int n, int8_t *const *A, const long *M,
                   const long *K)
{
    CHAIN_SWITCH(ref_flashgemm_multi_int8uint8int32, C, B, N, n)
}

}  // extern "C"
