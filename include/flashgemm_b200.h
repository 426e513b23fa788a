/* flashgemm-b200 extension API.
 *
 * Everything here is new relative to the reference (whose API is the four
 * symbols of flashgemm.h and the LibShalom entry points of libshalom.h): error
 * reporting, the semantics and FP32-algorithm switches, and entry points that
 * take device pointers and a CUDA stream. No torch types: plain pointers,
 * sizes and a stream handle passed as void* (a cudaStream_t; NULL means CUDA's
 * legacy default stream).
 */
#ifndef FLASHGEMM_B200_EXT_H
#define FLASHGEMM_B200_EXT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    FG_OK = 0,
    FG_ERR_INVALID = 1,     /* bad shape, pointer or argument */
    FG_ERR_UNSUPPORTED = 2, /* valid for the reference but not handled here */
    FG_ERR_CUDA = 3,        /* a CUDA runtime call failed */
    FG_ERR_NO_DEVICE = 4,   /* no usable sm_100 device */
    FG_ERR_TIMEOUT = 5,     /* a kernel's bounded pipeline wait ran out */
    FG_ERR_NOMEM = 6        /* device scratch allocation failed */
} fg_status;

/* Status and message of the last call made on this host thread. */
int fg_last_status(void);
const char *fg_last_error(void);

/* Chain semantics.
 * FG_SEM_REF  (default): what the reference computes. BF16 and INT8 chains
 *   apply the reference's between-stage panel permutation (its stage output is
 *   stored row-major and re-read as K-pair / K-quad interleaved packed B,
 *   multigemm/src/kernel_bf16.h:6-32 + :356-391, kernel_int8.h:6-50 +
 *   :329-385), INT8 tail rows 12*floor(M/12) <= m < 4*floor(M/4) use the
 *   reference's shifted k-quad pairing, and INT8 rows m >= 4*floor(M/4) of C
 *   are left untouched.
 * FG_SEM_MATH: the mathematical chain with the same narrowing points (BF16 RNE,
 *   INT8 signed saturation) and no permutation.
 * The environment variable FG_SEMANTICS=ref|math sets the initial value. */
enum { FG_SEM_REF = 0, FG_SEM_MATH = 1 };
void fg_set_semantics(int sem);
int fg_get_semantics(void);

/* FP32 GEMM algorithm, separately for the chain and for LibShalom SGEMM.
 * FG_F32_FFMA:   plain FP32 FMA on the CUDA cores, bit-identical to the
 *                reference (default for LibShalom_sgemm_mp).
 * FG_F32_3XTF32: split-precision 3xTF32 on the tensor cores: each operand
 *                x = hi + lo (both TF32, round to nearest even), product
 *                hi*hi + hi*lo + lo*hi accumulated in FP32 (default for the chain).
 * Environment: FG_F32_ALGO / FG_SGEMM_ALGO = ffma|3xtf32. */
enum { FG_F32_FFMA = 0, FG_F32_3XTF32 = 1 };
void fg_set_f32_algo(int algo);
int fg_get_f32_algo(void);
void fg_set_sgemm_algo(int algo);
int fg_get_sgemm_algo(void);

/* Element types of a chain. */
enum { FG_DT_F32 = 0, FG_DT_BF16 = 1, FG_DT_INT8 = 2 };

/* Chain on device memory of the current device, same shapes and semantics as
 * the flashgemm_multi_* entry points: A[i] is M[i] x K[i] with leading
 * dimension K[i], B is K[0] x N and C is M[n-1] x N, both with leading
 * dimension N. C is float (FG_DT_F32, FG_DT_BF16) or int32 (FG_DT_INT8).
 * Asynchronous with respect to the host: ordered after the work already on
 * `stream`, and work later put on `stream` is ordered after it. Returns a
 * fg_status; errors that only a kernel can see (bounded waits that ran out)
 * show up in fg_sync(). */
int fg_chain_dev(int dtype, void *C, const void *B, long N, int num_gemm, const void *const *A,
                 const long *M, const long *K, void *stream);

/* C = A * B on device memory (row-major, dense leading dimensions), with the
 * given FP32 algorithm (FG_F32_FFMA or FG_F32_3XTF32). Asynchronous like
 * fg_chain_dev. */
int fg_sgemm_dev(float *C, const float *A, const float *B, long M, long N, long K, int algo,
                 void *stream);

/* Wait for all of the library's work on the current device and report any
 * kernel-side error since the last fg_sync (then cleared). */
int fg_sync(void);

/* Number of kernels this library has launched in this process (all devices).
 * Lets a benchmark count its own launches. */
unsigned long long fg_kernel_launches(void);

/* Per-launch device timing. While profiling is on, every kernel the library
 * launches on the current device is bracketed by CUDA events on the stream it
 * runs on. fg_profile_query sums, for one kernel class (or -1 for all), the
 * device time in ms, the number of launches and the algorithmic FLOPs
 * (2*M*N*K per GEMM stage). */
enum {
    FG_PK_TC_BF16 = 0,   /* tensor-core stage, BF16 */
    FG_PK_TC_I8 = 1,     /* tensor-core stage, INT8 */
    FG_PK_TC_TF32X3 = 2, /* tensor-core stage, 3xTF32 */
    FG_PK_FFMA = 3,      /* CUDA-core FP32 GEMM */
    FG_PK_AUX = 4        /* splits, weight preparation */
};
int fg_profile_begin(void);
int fg_profile_end(void);
int fg_profile_query(int kind, double *total_ms, unsigned long long *launches, double *flops);

/* Library version string. */
const char *fg_version(void);

#ifdef __cplusplus
}
#endif

#endif
