// Internal interface between the host shim (fg_api.cpp) and the CUDA kernels.
// Not installed; the public C ABI is in include/.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace fg {

// How a tensor-core GEMM stage writes its result.
enum EpiKind : int {
    EPI_F32 = 0,       // final stage, FP32 C (BF16 / TF32 chains, SGEMM)
    EPI_S32 = 1,       // final stage, int32 C (INT8 chain)
    EPI_BF16 = 2,      // between stages: FP32 -> BF16 (RNE), optional panel permutation
    EPI_S8 = 3,        // between stages: int32 -> int8 (saturate), optional panel permutation
    EPI_TF32SPLIT = 4  // between stages: FP32 -> (hi, lo) TF32 pair for the next 3xTF32 stage
};

enum OperandKind : int { OP_BF16 = 0, OP_I8 = 1, OP_TF32X3 = 2 };

// One GEMM stage D[M x N] = W[M x K] * X[K x N]; W row-major with leading
// dimension ld_w, X row-major with leading dimension ld_x (both in elements).
struct StageArgs {
    int op;            // OperandKind
    int M, N, K;
    const void *w;     // weights (TF32X3: hi part)
    const void *w_lo;  // TF32X3: lo part (same ld)
    long ld_w;
    const void *x;     // activations (TF32X3: hi part)
    const void *x_lo;  // TF32X3: lo part (same ld)
    long ld_x;
    int epi;           // EpiKind
    void *out;         // C, or the next stage's activations (TF32SPLIT: hi)
    void *out_lo;      // TF32SPLIT: lo
    long ld_out;
    int permute;       // 1: apply the reference's panel permutation (EPI_BF16 / EPI_S8)
    int m_written;     // rows >= m_written are not stored (INT8 reference semantics)
    int tail_lo;       // INT8 reference tail rows [tail_lo, tail_hi): their weights come from
    int tail_hi;       //   w_tail (rows tail_row0 .. M-1, pre-shifted by one k-quad, first
    const void *w_tail;//   quad kept at [K, K + 4) for the epilogue's correction term)
    long ld_w_tail;
    int tail_row0;
    int kchunk;        // TF32X3: k-blocks (of 32) per FP32 promotion of the partial sum
    int tma_store;     // set by the launchers: the epilogue writes `out` with TMA bulk stores
    int *status;       // device status word (0 = ok)
};

cudaError_t launch_tc_stage(const StageArgs &a, int num_sms, cudaStream_t s);

// A whole BF16 or INT8 chain (stages[0..n) with the same op and N) in one
// cooperative persistent launch; `done` holds n * ceil(N / 256) zeroed ints.
// Returns cudaErrorNotSupported (nothing launched) where the device cannot
// run it; the caller then launches the stages one by one.
// trace (optional, else null): chain_trace_fields() %globaltimer stamps per (item, CTA).
cudaError_t launch_tc_chain(const StageArgs *stages, int n, int *done, int *status,
                            unsigned long long *trace, int num_sms, cudaStream_t s);
int chain_max_stages();
int chain_trace_fields();

// Several chains of one op in one launch: stage i reads the output of stage
// prev[i] (-1: a chain's first stage; prev[i] < i). `done` holds
// sum_i ceil(N_i / 256) zeroed ints; ext_dev (device memory of
// chain_group_table_bytes(n, work entries) bytes, or null) holds the stage table
// and schedule when they do not fit in the kernel parameters.
cudaError_t launch_tc_group(const StageArgs *stages, const int *prev, int n, int *done,
                            int *status, unsigned long long *trace, void *ext_dev, int num_sms,
                            cudaStream_t s);
size_t chain_group_table_bytes(int nstages, long items);

// Plain FP32 SGEMM on CUDA cores: C = A * B, one FMA per k in increasing k;
// with kblock > 0 each block of kblock k is summed from zero and added to C.
struct FfmaArgs {
    int M, N, K;
    const float *A; long lda;
    const float *B; long ldb;
    float *C; long ldc;
    int kblock;
};
cudaError_t launch_ffma_sgemm(const FfmaArgs &a, int num_sms, cudaStream_t s);

// FP32 -> (hi, lo) TF32 split of a rows x cols matrix (leading dims ld_in / ld_out).
cudaError_t launch_split_tf32(const float *in, long ld_in, float *hi, float *lo, long ld_out,
                              long rows, long cols, cudaStream_t s);

// INT8 weight preparation: copies W (M x K, ld_in) into dst (ld_out >= K + 4,
// a multiple of 16), shifting rows [tail_lo, tail_hi) left by one k-quad
// (zero-filling the last quad) and keeping their first quad at [K, K + 4).
cudaError_t launch_prep_int8_weights(const int8_t *src, long ld_in, uint8_t *dst, long ld_out,
                                     long M, long K, long tail_lo, long tail_hi,
                                     cudaStream_t s);

// The same preparation for up to 8 matrices in one launch.
struct PrepJob {
    const int8_t *src;
    long ld_in;
    uint8_t *dst;
    long ld_out;
    long M, K, tail_lo, tail_hi;
};
struct PrepJobs {
    PrepJob job[8];
    int n;
};
cudaError_t launch_prep_int8_jobs(const PrepJobs &jobs, cudaStream_t s);

// Fill `count` 32-bit words with `value`.
cudaError_t launch_fill_u32(uint32_t *dst, size_t count, uint32_t value, cudaStream_t s);

}  // namespace fg
