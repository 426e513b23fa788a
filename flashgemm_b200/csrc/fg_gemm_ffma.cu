// Plain FP32 SGEMM on the CUDA cores: C = A * B, row-major.
//
// Each output is one FP32 fused multiply-add per k in increasing k, the
// arithmetic of the reference's vfmadd231ps register tiles
// (singlegemm/src/kernel.h:8, multigemm/src/kernel_f32.h:3), so results are
// bit-identical to the reference's. With kblock > 0, K is cut into blocks of
// kblock: each block is summed from zero and then added into the result, as
// singlegemm's GEMM_K = 2048 blocking does (singlegemm/src/NN_mp.h:13 and its
// ADD_C step, singlegemm/src/kernel.h:384-400).
//
// Tiling: BM x BN block tile, BK = 8, TM x TN outputs per thread; A is staged
// transposed (k-major) and B as is, double-buffered in shared memory with the
// next tile prefetched into registers while the current one is consumed.
#include <cuda_runtime.h>

#include "fg_kernels.h"

namespace fg {

template <int BM, int BN, int TM, int TN, bool VEC>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
    ffma_sgemm_kernel(const FfmaArgs p)
{
    constexpr int BK = 8;
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr int A_LOADS = BM * BK / NT;  // elements per thread per tile
    constexpr int B_LOADS = BK * BN / NT;
    static_assert(A_LOADS % 4 == 0 && B_LOADS % 4 == 0, "vector tiling");
    __shared__ __align__(16) float As[2][BK][BM];
    __shared__ __align__(16) float Bs[2][BK][BN];

    const int tid = threadIdx.x;
    const int tx = tid % (BN / TN);
    const int ty = tid / (BN / TN);
    const int m0 = blockIdx.y * BM;
    const int n0 = blockIdx.x * BN;
    const int M = p.M, N = p.N, K = p.K;

    // Load mapping. A: thread handles A_LOADS consecutive k of one row;
    // B: thread handles B_LOADS consecutive n of one k row.
    constexpr int A_TPR = BK / A_LOADS;  // threads per A row
    const int a_row = tid / A_TPR;
    const int a_k = (tid % A_TPR) * A_LOADS;
    constexpr int B_TPR = BN / B_LOADS;
    const int b_row = tid / B_TPR;
    const int b_n = (tid % B_TPR) * B_LOADS;

    float ra[A_LOADS], rb[B_LOADS];

    auto load_tile = [&](int k0) {
        const int gm = m0 + a_row;
#pragma unroll
        for (int v = 0; v < A_LOADS; v += 4) {
            const int gk = k0 + a_k + v;
            if (VEC && gm < M && gk + 3 < K) {
                float4 t = *reinterpret_cast<const float4 *>(p.A + (size_t)gm * p.lda + gk);
                ra[v] = t.x; ra[v + 1] = t.y; ra[v + 2] = t.z; ra[v + 3] = t.w;
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    ra[v + u] = (gm < M && gk + u < K) ? p.A[(size_t)gm * p.lda + gk + u] : 0.f;
            }
        }
        const int gk = k0 + b_row;
#pragma unroll
        for (int v = 0; v < B_LOADS; v += 4) {
            const int gn = n0 + b_n + v;
            if (VEC && gk < K && gn + 3 < N) {
                float4 t = *reinterpret_cast<const float4 *>(p.B + (size_t)gk * p.ldb + gn);
                rb[v] = t.x; rb[v + 1] = t.y; rb[v + 2] = t.z; rb[v + 3] = t.w;
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    rb[v + u] = (gk < K && gn + u < N) ? p.B[(size_t)gk * p.ldb + gn + u] : 0.f;
            }
        }
    };
    auto store_tile = [&](int buf) {
#pragma unroll
        for (int v = 0; v < A_LOADS; ++v) As[buf][a_k + v][a_row] = ra[v];
#pragma unroll
        for (int v = 0; v < B_LOADS; v += 4)
            *reinterpret_cast<float4 *>(&Bs[buf][b_row][b_n + v]) =
                make_float4(rb[v], rb[v + 1], rb[v + 2], rb[v + 3]);
    };

    float acc[TM][TN];
    float sum[TM][TN];
    const int kblock = (p.kblock > 0 && p.kblock < K) ? p.kblock : K;

    for (int kb0 = 0; kb0 < K; kb0 += kblock) {
        const int kb1 = min(kb0 + kblock, K);
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN; ++j) acc[i][j] = 0.f;

        load_tile(kb0);
        store_tile(0);
        __syncthreads();
        int buf = 0;
        for (int k0 = kb0; k0 < kb1; k0 += BK) {
            const bool more = k0 + BK < kb1;
            if (more) load_tile(k0 + BK);
            const int kend = min(BK, kb1 - k0);
#pragma unroll
            for (int kk = 0; kk < BK; ++kk) {
                if (kk < kend) {
                    float a[TM], b[TN];
#pragma unroll
                    for (int i = 0; i < TM; i += 4) {
                        float4 t = *reinterpret_cast<const float4 *>(&As[buf][kk][ty * TM + i]);
                        a[i] = t.x; a[i + 1] = t.y; a[i + 2] = t.z; a[i + 3] = t.w;
                    }
#pragma unroll
                    for (int j = 0; j < TN; j += 4) {
                        float4 t = *reinterpret_cast<const float4 *>(&Bs[buf][kk][tx * TN + j]);
                        b[j] = t.x; b[j + 1] = t.y; b[j + 2] = t.z; b[j + 3] = t.w;
                    }
#pragma unroll
                    for (int i = 0; i < TM; ++i)
#pragma unroll
                        for (int j = 0; j < TN; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
                }
            }
            if (more) {
                store_tile(buf ^ 1);
                __syncthreads();
                buf ^= 1;
            }
        }
        __syncthreads();  // buffers are refilled by the next K block
        if (kb0 == 0) {
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) sum[i][j] = acc[i][j];
        } else {
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) sum[i][j] = sum[i][j] + acc[i][j];
        }
    }
    if (K == 0) {
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN; ++j) sum[i][j] = 0.f;
    }

#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int gm = m0 + ty * TM + i;
        if (gm >= M) continue;
        float *c = p.C + (size_t)gm * p.ldc;
#pragma unroll
        for (int j = 0; j < TN; j += 4) {
            const int gn = n0 + tx * TN + j;
            if (VEC && gn + 3 < N) {
                *reinterpret_cast<float4 *>(c + gn) =
                    make_float4(sum[i][j], sum[i][j + 1], sum[i][j + 2], sum[i][j + 3]);
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (gn + u < N) c[gn + u] = sum[i][j + u];
            }
        }
    }
}

template <int BM, int BN, int TM, int TN>
static cudaError_t launch_cfg(const FfmaArgs &a, bool vec, cudaStream_t s)
{
    dim3 grid((a.N + BN - 1) / BN, (a.M + BM - 1) / BM);
    dim3 block((BM / TM) * (BN / TN));
    if (vec)
        ffma_sgemm_kernel<BM, BN, TM, TN, true><<<grid, block, 0, s>>>(a);
    else
        ffma_sgemm_kernel<BM, BN, TM, TN, false><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_ffma_sgemm(const FfmaArgs &a, int num_sms, cudaStream_t s)
{
    if (a.M <= 0 || a.N <= 0) return cudaSuccess;
    const bool vec = ((a.lda | a.ldb | a.ldc) % 4 == 0) &&
                     (((uintptr_t)a.A | (uintptr_t)a.B | (uintptr_t)a.C) % 16 == 0);
    // Largest tile that still gives every SM a block; small problems drop to
    // 64 x 64 tiles so that more of the 148 SMs have work.
    const long tiles128 = (long)((a.M + 127) / 128) * ((a.N + 127) / 128);
    if (tiles128 >= num_sms) return launch_cfg<128, 128, 8, 8>(a, vec, s);
    const long tiles64 = (long)((a.M + 127) / 128) * ((a.N + 63) / 64);
    if (tiles64 >= num_sms) return launch_cfg<128, 64, 8, 8>(a, vec, s);
    return launch_cfg<64, 64, 4, 8>(a, vec, s);
}

}  // namespace fg
