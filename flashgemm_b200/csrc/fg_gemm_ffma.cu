// Plain FP32 SGEMM on the CUDA cores: C = A * B, row-major.
//
// Each output is one FP32 fused multiply-add per k in increasing k, the
// arithmetic of the reference's vfmadd231ps register tiles
// (singlegemm/src/kernel.h:8, multigemm/src/kernel_f32.h:3), so results are
// bit-identical to the reference's. With kblock > 0 and K > kblock, K is cut
// into blocks of kblock: each block is summed from zero and then added into
// the result, as singlegemm's GEMM_K = 2048 blocking does
// (singlegemm/src/NN_mp.h:13 and its ADD_C step, singlegemm/src/kernel.h:384-400).
//
// Tiling: BM x BN block tile, BK-deep k slices, TM x TN outputs per thread
// held as float4 fragments spread over the tile (rows ty*4 + i*BM/(TM/4),
// columns tx*4 + j*BN/(TN/4)) so that a warp's float4 shared-memory reads fall
// on distinct banks; A is staged transposed (k-major) and B as is,
// double-buffered in shared memory with the next slice prefetched into
// registers while the current one is consumed.
#include <cuda_runtime.h>

#include <cstdlib>

#include "fg_kernels.h"

namespace fg {

// One BM x BN output tile at (m0, n0); As / Bs are the block's double buffers.
template <int BM, int BN, int BK, int TM, int TN, bool VEC, bool KSPLIT>
__device__ __forceinline__ void ffma_tile(const FfmaArgs &p, int m0, int n0,
                                          float (*As)[BK][BM], float (*Bs)[BK][BN])
{
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr int A_LOADS = BM * BK / NT;  // elements per thread per slice
    constexpr int B_LOADS = BK * BN / NT;
    static_assert(A_LOADS % 4 == 0 && B_LOADS % 4 == 0, "vector tiling");
    static_assert(TM % 4 == 0 && TN % 4 == 0, "float4 fragments");

    const int tid = threadIdx.x;
    const int tx = tid % (BN / TN);
    const int ty = tid / (BN / TN);
    const int M = p.M, N = p.N, K = p.K;

    // A: a thread loads A_LOADS consecutive k of one row; B: B_LOADS consecutive n of one k row.
    constexpr int A_TPR = BK / A_LOADS;
    const int a_row = tid / A_TPR;
    const int a_k = (tid % A_TPR) * A_LOADS;
    constexpr int B_TPR = BN / B_LOADS;
    const int b_row = tid / B_TPR;
    const int b_n = (tid % B_TPR) * B_LOADS;

    // Fragment placement: rows ty*4 + {0..3} + i*(BM/2) for the two halves of TM,
    // columns tx*4 + {0..3} + j*(BN/2) for the two halves of TN.
    constexpr int HM = TM / 4, HN = TN / 4;  // float4 fragments per thread per dimension
    float ra[A_LOADS], rb[B_LOADS];

    auto load_slice = [&](int k0) {
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
    auto store_slice = [&](int buf) {
#pragma unroll
        for (int v = 0; v < A_LOADS; ++v) As[buf][a_k + v][a_row] = ra[v];
#pragma unroll
        for (int v = 0; v < B_LOADS; v += 4)
            *reinterpret_cast<float4 *>(&Bs[buf][b_row][b_n + v]) =
                make_float4(rb[v], rb[v + 1], rb[v + 2], rb[v + 3]);
    };

    float acc[TM][TN];
    float sum[KSPLIT ? TM : 1][KSPLIT ? TN : 1];
    const int kblock = (KSPLIT && p.kblock > 0 && p.kblock < K) ? p.kblock : K;

    for (int kb0 = 0; kb0 < K; kb0 += kblock) {
        const int kb1 = min(kb0 + kblock, K);
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN; ++j) acc[i][j] = 0.f;

        load_slice(kb0);
        store_slice(0);
        __syncthreads();
        int buf = 0;
        for (int k0 = kb0; k0 < kb1; k0 += BK) {
            const bool more = k0 + BK < kb1;
            if (more) load_slice(k0 + BK);
            // a slice past K holds zeros for both operands; skip those k so that
            // no extra rounding step touches the sum
            const int kend = min(BK, kb1 - k0);
            if (kend == BK) {
#pragma unroll
                for (int kk = 0; kk < BK; ++kk) {
                    float a[TM], b[TN];
#pragma unroll
                    for (int i = 0; i < HM; ++i) {
                        float4 t = *reinterpret_cast<const float4 *>(
                            &As[buf][kk][ty * 4 + i * (BM / HM)]);
                        a[4 * i] = t.x; a[4 * i + 1] = t.y; a[4 * i + 2] = t.z; a[4 * i + 3] = t.w;
                    }
#pragma unroll
                    for (int j = 0; j < HN; ++j) {
                        float4 t = *reinterpret_cast<const float4 *>(
                            &Bs[buf][kk][tx * 4 + j * (BN / HN)]);
                        b[4 * j] = t.x; b[4 * j + 1] = t.y; b[4 * j + 2] = t.z; b[4 * j + 3] = t.w;
                    }
#pragma unroll
                    for (int i = 0; i < TM; ++i)
#pragma unroll
                        for (int j = 0; j < TN; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
                }
            } else {
                for (int kk = 0; kk < kend; ++kk) {
                    float a[TM], b[TN];
#pragma unroll
                    for (int i = 0; i < HM; ++i) {
                        float4 t = *reinterpret_cast<const float4 *>(
                            &As[buf][kk][ty * 4 + i * (BM / HM)]);
                        a[4 * i] = t.x; a[4 * i + 1] = t.y; a[4 * i + 2] = t.z; a[4 * i + 3] = t.w;
                    }
#pragma unroll
                    for (int j = 0; j < HN; ++j) {
                        float4 t = *reinterpret_cast<const float4 *>(
                            &Bs[buf][kk][tx * 4 + j * (BN / HN)]);
                        b[4 * j] = t.x; b[4 * j + 1] = t.y; b[4 * j + 2] = t.z; b[4 * j + 3] = t.w;
                    }
#pragma unroll
                    for (int i = 0; i < TM; ++i)
#pragma unroll
                        for (int j = 0; j < TN; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
                }
            }
            if (more) {
                store_slice(buf ^ 1);
                __syncthreads();
                buf ^= 1;
            }
        }
        if constexpr (KSPLIT) {
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
    }
    if (K == 0) {
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN; ++j) acc[i][j] = 0.f;
    }

#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int gm = m0 + ty * 4 + (i / 4) * (BM / HM) + (i % 4);
        if (gm >= M) continue;
        float *c = p.C + (size_t)gm * p.ldc;
#pragma unroll
        for (int j = 0; j < HN; ++j) {
            const int gn = n0 + tx * 4 + j * (BN / HN);
            float r[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if constexpr (KSPLIT)
                    r[u] = K > 0 ? sum[i][4 * j + u] : 0.f;
                else
                    r[u] = acc[i][4 * j + u];
            }
            if (VEC && gn + 3 < N) {
                *reinterpret_cast<float4 *>(c + gn) = make_float4(r[0], r[1], r[2], r[3]);
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (gn + u < N) c[gn + u] = r[u];
            }
        }
    }
}

template <int BM, int BN, int BK, int TM, int TN, bool VEC, bool KSPLIT>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
    ffma_sgemm_kernel(const FfmaArgs p)
{
    __shared__ __align__(16) float As[2][BK][BM];
    __shared__ __align__(16) float Bs[2][BK][BN];
    ffma_tile<BM, BN, BK, TM, TN, VEC, KSPLIT>(p, blockIdx.y * BM, blockIdx.x * BN, As, Bs);
}

// Many independent SGEMMs: CTA b works on job j with tile0[j] <= b < tile0[j + 1].
template <int BM, int BN, int BK, int TM, int TN>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
    ffma_group_kernel(const FfmaJob *__restrict__ jobs, int njobs)
{
    __shared__ __align__(16) float As[2][BK][BM];
    __shared__ __align__(16) float Bs[2][BK][BN];
    const int b = blockIdx.x;
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].tile0 <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    const FfmaJob &j = jobs[lo];
    const int t = b - j.tile0;
    FfmaArgs p;
    p.M = j.M; p.N = j.N; p.K = j.K;
    p.A = j.A; p.lda = j.lda;
    p.B = j.B; p.ldb = j.ldb;
    p.C = j.C; p.ldc = j.ldc;
    p.kblock = 0;
    const int m0 = (t / j.tiles_n) * BM, n0 = (t % j.tiles_n) * BN;
    if (j.vec)
        ffma_tile<BM, BN, BK, TM, TN, true, false>(p, m0, n0, As, Bs);
    else
        ffma_tile<BM, BN, BK, TM, TN, false, false>(p, m0, n0, As, Bs);
}

int ffma_group_tile(int big) { return big ? 128 : 64; }

cudaError_t launch_ffma_group(const FfmaJob *jobs_dev, int njobs, int total_tiles, int big,
                              cudaStream_t s)
{
    if (njobs < 1 || total_tiles < 1) return cudaSuccess;
    if (big)
        ffma_group_kernel<128, 128, 16, 8, 8><<<total_tiles, 256, 0, s>>>(jobs_dev, njobs);
    else
        ffma_group_kernel<64, 64, 16, 4, 8><<<total_tiles, 128, 0, s>>>(jobs_dev, njobs);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ 8 x 8 per thread
//
// The shape of small SGEMMs (1024^3 has 256 tiles of 64 x 64 for 148 SMs):
// 64 x 64 tiles of 64 threads, 8 x 8 outputs per thread in four 4 x 4
// quadrants (rows ty*4 + {0, 32}, columns tx*4 + {0, 32}), so that a thread
// loads 8 + 8 values from shared memory per k for 64 multiply-adds (half the
// shared-memory traffic per FMA of 4 x 8), fragments of k + 1 loaded while k
// computes. The multiply-adds go in pairs (fma.rn.f32x2: two IEEE
// round-to-nearest FMAs per instruction, each exactly an fmaf), so every
// output is still one FMA per k in increasing k. Staging: the next 16-deep k
// slice is read from global memory into registers while the current one is
// consumed; A is stored transposed (k-major), B row by row, each quarter-warp
// writing 128 contiguous bytes.

__device__ __forceinline__ unsigned long long pack2(float lo, float hi)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}

__device__ __forceinline__ void unpack2(unsigned long long v, float &lo, float &hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}

// d (two lanes) = a * b + d, each lane one round-to-nearest FMA
__device__ __forceinline__ void ffma2(unsigned long long &d, unsigned long long a,
                                      unsigned long long b)
{
    asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(d) : "l"(a), "l"(b));
}

template <bool KSPLIT>
__global__ void __launch_bounds__(64) ffma_sgemm_8x8_kernel(const FfmaArgs p)
{
    constexpr int BM = 64, BN = 64, BK = 16;
    __shared__ __align__(16) float As[2][BK][BM];
    __shared__ __align__(16) float Bs[2][BK][BN];
    const int tid = threadIdx.x;
    const int tx = tid & 7, ty = tid >> 3;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int M = p.M, N = p.N, K = p.K;

    float4 ra[4], rb[4];
    // A: row m0 + tid, 16 k; B: rows tid / 16 + 4 v, 4 columns at (tid % 16) * 4
    auto load_slice = [&](int k0) {
        const int gm = m0 + tid;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int gk = k0 + 4 * v;
            if (gm < M && gk + 3 < K) {
                ra[v] = *reinterpret_cast<const float4 *>(p.A + (size_t)gm * p.lda + gk);
            } else {
                const float *a = p.A + (size_t)gm * p.lda;
                ra[v].x = (gm < M && gk < K) ? a[gk] : 0.f;
                ra[v].y = (gm < M && gk + 1 < K) ? a[gk + 1] : 0.f;
                ra[v].z = (gm < M && gk + 2 < K) ? a[gk + 2] : 0.f;
                ra[v].w = (gm < M && gk + 3 < K) ? a[gk + 3] : 0.f;
            }
        }
        const int gn = n0 + (tid & 15) * 4;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int gk = k0 + (tid >> 4) + 4 * v;
            if (gk < K && gn + 3 < N) {
                rb[v] = *reinterpret_cast<const float4 *>(p.B + (size_t)gk * p.ldb + gn);
            } else {
                const float *b = p.B + (size_t)gk * p.ldb;
                rb[v].x = (gk < K && gn < N) ? b[gn] : 0.f;
                rb[v].y = (gk < K && gn + 1 < N) ? b[gn + 1] : 0.f;
                rb[v].z = (gk < K && gn + 2 < N) ? b[gn + 2] : 0.f;
                rb[v].w = (gk < K && gn + 3 < N) ? b[gn + 3] : 0.f;
            }
        }
    };
    auto store_slice = [&](int buf) {
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            As[buf][4 * v + 0][tid] = ra[v].x;
            As[buf][4 * v + 1][tid] = ra[v].y;
            As[buf][4 * v + 2][tid] = ra[v].z;
            As[buf][4 * v + 3][tid] = ra[v].w;
            *reinterpret_cast<float4 *>(&Bs[buf][(tid >> 4) + 4 * v][(tid & 15) * 4]) = rb[v];
        }
    };

    unsigned long long acc[8][4];  // row i, column pairs {0,1}, {2,3} of each quadrant
    unsigned long long sum[KSPLIT ? 8 : 1][KSPLIT ? 4 : 1];
    const int kblock = (KSPLIT && p.kblock > 0 && p.kblock < K) ? p.kblock : K;

    for (int kb0 = 0; kb0 < K; kb0 += kblock) {
        const int kb1 = min(kb0 + kblock, K);
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = 0ull;

        load_slice(kb0);
        store_slice(0);
        __syncthreads();
        int buf = 0;
        for (int k0 = kb0; k0 < kb1; k0 += BK) {
            const bool more = k0 + BK < kb1;
            if (more) load_slice(k0 + BK);
            // a slice past K holds zeros for both operands; its k are skipped so
            // that no extra rounding step touches the sums
            const int kend = min(BK, kb1 - k0);
            auto step = [&](int kk) {
                const float4 a0 = *reinterpret_cast<const float4 *>(&As[buf][kk][ty * 4]);
                const float4 a1 = *reinterpret_cast<const float4 *>(&As[buf][kk][ty * 4 + 32]);
                const float4 b0 = *reinterpret_cast<const float4 *>(&Bs[buf][kk][tx * 4]);
                const float4 b1 = *reinterpret_cast<const float4 *>(&Bs[buf][kk][tx * 4 + 32]);
                const unsigned long long bp[4] = {pack2(b0.x, b0.y), pack2(b0.z, b0.w),
                                                  pack2(b1.x, b1.y), pack2(b1.z, b1.w)};
                const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const unsigned long long ap = pack2(a[i], a[i]);
#pragma unroll
                    for (int j = 0; j < 4; ++j) ffma2(acc[i][j], ap, bp[j]);
                }
            };
            if (kend == BK) {
#pragma unroll
                for (int kk = 0; kk < BK; ++kk) step(kk);
            } else {
                for (int kk = 0; kk < kend; ++kk) step(kk);
            }
            if (more) {
                store_slice(buf ^ 1);
                __syncthreads();
                buf ^= 1;
            }
        }
        if constexpr (KSPLIT) {
            __syncthreads();  // buffers are refilled by the next K block
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    if (kb0 == 0) {
                        sum[i][j] = acc[i][j];
                    } else {
                        float s0, s1, a0, a1;
                        unpack2(sum[i][j], s0, s1);
                        unpack2(acc[i][j], a0, a1);
                        sum[i][j] = pack2(s0 + a0, s1 + a1);
                    }
                }
        }
    }

#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int gm = m0 + ty * 4 + (i / 4) * 32 + (i % 4);
        if (gm >= M) continue;
        float *c = p.C + (size_t)gm * p.ldc;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int gn = n0 + tx * 4 + h * 32;
            float r[4];
            unsigned long long v0 = KSPLIT ? sum[i][2 * h] : acc[i][2 * h];
            unsigned long long v1 = KSPLIT ? sum[i][2 * h + 1] : acc[i][2 * h + 1];
            if (K == 0) v0 = v1 = 0ull;
            unpack2(v0, r[0], r[1]);
            unpack2(v1, r[2], r[3]);
            if (gn + 3 < N) {
                *reinterpret_cast<float4 *>(c + gn) = make_float4(r[0], r[1], r[2], r[3]);
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (gn + u < N) c[gn + u] = r[u];
            }
        }
    }
}

static cudaError_t launch_8x8(const FfmaArgs &a, cudaStream_t s)
{
    dim3 grid((a.N + 63) / 64, (a.M + 63) / 64);
    if (a.kblock > 0 && a.kblock < a.K)
        ffma_sgemm_8x8_kernel<true><<<grid, 64, 0, s>>>(a);
    else
        ffma_sgemm_8x8_kernel<false><<<grid, 64, 0, s>>>(a);
    return cudaGetLastError();
}

template <int BM, int BN, int BK, int TM, int TN>
static cudaError_t launch_cfg(const FfmaArgs &a, bool vec, cudaStream_t s)
{
    dim3 grid((a.N + BN - 1) / BN, (a.M + BM - 1) / BM);
    dim3 block((BM / TM) * (BN / TN));
    const bool split = a.kblock > 0 && a.kblock < a.K;
    if (vec) {
        if (split)
            ffma_sgemm_kernel<BM, BN, BK, TM, TN, true, true><<<grid, block, 0, s>>>(a);
        else
            ffma_sgemm_kernel<BM, BN, BK, TM, TN, true, false><<<grid, block, 0, s>>>(a);
    } else {
        if (split)
            ffma_sgemm_kernel<BM, BN, BK, TM, TN, false, true><<<grid, block, 0, s>>>(a);
        else
            ffma_sgemm_kernel<BM, BN, BK, TM, TN, false, false><<<grid, block, 0, s>>>(a);
    }
    return cudaGetLastError();
}

cudaError_t launch_ffma_sgemm(const FfmaArgs &a, int num_sms, cudaStream_t s)
{
    if (a.M <= 0 || a.N <= 0) return cudaSuccess;
    if (a.kblock > 0 && a.kblock % 16) return cudaErrorInvalidValue;  // K blocks end on slices
    const bool vec = ((a.lda | a.ldb | a.ldc) % 4 == 0) &&
                     (((uintptr_t)a.A | (uintptr_t)a.B | (uintptr_t)a.C) % 16 == 0);
    // FG_FFMA_CFG forces one tile configuration (0..8). By default 128 x 128 x 16
    // tiles when there are at least two per SM, else 64 x 64 x 16 with 8 x 8 per
    // thread (measured on B200 with 4 x 8 per thread: 1024^3 25.9 TFLOP/s with
    // 64 x 64 vs 17.8 with 128 x 128; 4096^3 38.4 with 128 x 128 x 16).
    static const int forced = [] {
        const char *v = getenv("FG_FFMA_CFG");
        return v ? atoi(v) : -1;
    }();
    const long t128 = (long)((a.M + 127) / 128) * ((a.N + 127) / 128);
    const long t12864 = (long)((a.M + 127) / 128) * ((a.N + 63) / 64);
    int cfg = forced;
    if (cfg < 0) cfg = t128 >= 2l * num_sms ? 5 : (vec ? 8 : 2);
    (void)t12864;
    switch (cfg) {
    case 8:  // 64 x 64 x 16, 8 x 8 per thread (vector rows and pointers only)
        if (vec) return launch_8x8(a, s);
        return launch_cfg<64, 64, 16, 4, 8>(a, vec, s);
    case 0: return launch_cfg<128, 128, 8, 8, 8>(a, vec, s);   // 256 threads
    case 1: return launch_cfg<128, 64, 8, 8, 8>(a, vec, s);    // 128 threads
    case 2: return launch_cfg<64, 64, 16, 4, 8>(a, vec, s);    // 128 threads
    case 3: return launch_cfg<64, 128, 8, 8, 8>(a, vec, s);    // 128 threads
    case 4: return launch_cfg<64, 64, 32, 4, 8>(a, vec, s);    // 128 threads
    case 5: return launch_cfg<128, 128, 16, 8, 8>(a, vec, s);  // 256 threads
    case 6: return launch_cfg<64, 32, 32, 4, 4>(a, vec, s);    // 128 threads
    default: return launch_cfg<128, 64, 32, 8, 8>(a, vec, s);  // 128 threads
    }
}

}  // namespace fg
