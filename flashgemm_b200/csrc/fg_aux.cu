// Bandwidth-bound helper kernels around the GEMM stages: the FP32 -> TF32
// hi/lo split that feeds 3xTF32 stages, and the INT8 weight preparation that
// carries the reference's tail-row behaviour into the tensor-core path.
#include <cuda_runtime.h>

#include "fg_kernels.h"

namespace fg {

__device__ __forceinline__ float tf32_rne(float f)
{
    uint32_t u = __float_as_uint(f);
    if ((u & 0x7f800000u) == 0x7f800000u) return f;
    u += 0xfffu + ((u >> 13) & 1u);
    return __uint_as_float(u & 0xffffe000u);
}

// x = hi + lo + r with hi = rne_tf32(x), lo = rne_tf32(x - hi), |r| <= 2^-22 |x|.
__global__ void split_tf32_kernel(const float *__restrict__ in, long ld_in, float *__restrict__ hi,
                                  float *__restrict__ lo, long ld_out, long rows, long cols)
{
    const long total = rows * cols;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
         i += (long)gridDim.x * blockDim.x) {
        const long r = i / cols, c = i - r * cols;
        const float x = in[r * ld_in + c];
        const float h = tf32_rne(x);
        hi[r * ld_out + c] = h;
        lo[r * ld_out + c] = tf32_rne(x - h);
    }
}

cudaError_t launch_split_tf32(const float *in, long ld_in, float *hi, float *lo, long ld_out,
                              long rows, long cols, cudaStream_t s)
{
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    const long total = rows * cols;
    long blocks = (total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    split_tf32_kernel<<<(unsigned)blocks, 256, 0, s>>>(in, ld_in, hi, lo, ld_out, rows, cols);
    return cudaGetLastError();
}

// Many splits in one launch: blockIdx.y = job.
__global__ void split_tf32_jobs_kernel(const SplitJob *__restrict__ jobs)
{
    const SplitJob j = jobs[blockIdx.y];
    const long total = j.rows * j.cols;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
         i += (long)gridDim.x * blockDim.x) {
        const long r = i / j.cols, c = i - r * j.cols;
        const float x = j.in[r * j.ld_in + c];
        const float h = tf32_rne(x);
        j.hi[r * j.ld_out + c] = h;
        j.lo[r * j.ld_out + c] = tf32_rne(x - h);
    }
}

cudaError_t launch_split_tf32_jobs(const SplitJob *jobs_dev, int njobs, long max_elems,
                                   cudaStream_t s)
{
    if (njobs < 1 || max_elems < 1) return cudaSuccess;
    if (njobs > 65535) return cudaErrorInvalidValue;
    long blocks = (max_elems + 255) / 256;
    if (blocks > 148 * 4) blocks = 148 * 4;
    split_tf32_jobs_kernel<<<dim3((unsigned)blocks, (unsigned)njobs), 256, 0, s>>>(jobs_dev);
    return cudaGetLastError();
}

// Rows m in [tail_lo, tail_hi) of the reference's INT8 chain meet activation
// k-quad max(s-1, 0) with weight k-quad s (multigemm/src/kernel_int8.h:405 vs
// :427, :590 vs :608). The prepared copy shifts those rows left by one quad,
// so a plain MMA yields sum_{s>=1} A_q(s) X_q(s-1); the missing A_q(0) X_q(0)
// term is added by the GEMM epilogue from the first quad kept at [K, K + 4).
// Other rows are copied unchanged; columns [K, ld_out) of them are zero.
// One thread writes 16 bytes (ld_out is a multiple of 16).
__global__ void prep_int8_weights_kernel(const int8_t *__restrict__ src, long ld_in,
                                         uint8_t *__restrict__ dst, long ld_out, long M, long K,
                                         long tail_lo, long tail_hi)
{
    const long per_row = ld_out / 16;
    const long total = M * per_row;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
         i += (long)gridDim.x * blockDim.x) {
        const long m = i / per_row, k0 = (i - m * per_row) * 16;
        const uint8_t *row = reinterpret_cast<const uint8_t *>(src) + m * ld_in;
        const bool tail = (m >= tail_lo && m < tail_hi);
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint32_t word = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const long k = k0 + 4 * q + b;
                uint8_t v = 0;
                if (tail) {
                    if (k < K - 4)
                        v = row[k + 4];
                    else if (k >= K && k < K + 4)
                        v = row[k - K];
                } else if (k < K) {
                    v = row[k];
                }
                word |= (uint32_t)v << (8 * b);
            }
            w[q] = word;
        }
        *reinterpret_cast<uint4 *>(dst + m * ld_out + k0) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

cudaError_t launch_prep_int8_weights(const int8_t *src, long ld_in, uint8_t *dst, long ld_out,
                                     long M, long K, long tail_lo, long tail_hi, cudaStream_t s)
{
    if (M <= 0) return cudaSuccess;
    if (ld_out % 16) return cudaErrorInvalidValue;
    const long total = M * (ld_out / 16);
    long blocks = (total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    prep_int8_weights_kernel<<<(unsigned)blocks, 256, 0, s>>>(src, ld_in, dst, ld_out, M, K,
                                                               tail_lo, tail_hi);
    return cudaGetLastError();
}

// Several preparations in one launch (blockIdx.y = job).
__global__ void prep_int8_jobs_kernel(const PrepJob *__restrict__ jobs_unused, PrepJobs jobs)
{
    const PrepJob &j = jobs.job[blockIdx.y];
    const long per_row = j.ld_out / 16;
    const long total = j.M * per_row;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
         i += (long)gridDim.x * blockDim.x) {
        const long m = i / per_row, k0 = (i - m * per_row) * 16;
        const uint8_t *row = reinterpret_cast<const uint8_t *>(j.src) + m * j.ld_in;
        const bool tail = (m >= j.tail_lo && m < j.tail_hi);
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint32_t word = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const long k = k0 + 4 * q + b;
                uint8_t v = 0;
                if (tail) {
                    if (k < j.K - 4)
                        v = row[k + 4];
                    else if (k >= j.K && k < j.K + 4)
                        v = row[k - j.K];
                } else if (k < j.K) {
                    v = row[k];
                }
                word |= (uint32_t)v << (8 * b);
            }
            w[q] = word;
        }
        *reinterpret_cast<uint4 *>(j.dst + m * j.ld_out + k0) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

cudaError_t launch_prep_int8_jobs(const PrepJobs &jobs, cudaStream_t s)
{
    if (jobs.n <= 0) return cudaSuccess;
    long most = 0;
    for (int i = 0; i < jobs.n; ++i) {
        if (jobs.job[i].ld_out % 16) return cudaErrorInvalidValue;
        const long t = jobs.job[i].M * (jobs.job[i].ld_out / 16);
        most = t > most ? t : most;
    }
    long blocks = (most + 255) / 256;
    if (blocks > 148 * 4) blocks = 148 * 4;
    if (blocks < 1) blocks = 1;
    prep_int8_jobs_kernel<<<dim3((unsigned)blocks, jobs.n), 256, 0, s>>>(nullptr, jobs);
    return cudaGetLastError();
}

__global__ void fill_u32_kernel(uint32_t *dst, size_t count, uint32_t value)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
         i += (size_t)gridDim.x * blockDim.x)
        dst[i] = value;
}

cudaError_t launch_fill_u32(uint32_t *dst, size_t count, uint32_t value, cudaStream_t s)
{
    if (count == 0) return cudaSuccess;
    size_t blocks = (count + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    fill_u32_kernel<<<(unsigned)blocks, 256, 0, s>>>(dst, count, value);
    return cudaGetLastError();
}

}  // namespace fg
