// Tensor-core GEMM stage for sm_100a: D[M x N] = W[M x K] * X[K x N].
//
// Orientation. The reference computes C = A_n*(...*(A_1*B)) with A_i (M_i x K_i)
// and B (K_1 x N) row-major (multigemm/src/flashgemm.h:17-25). Here a stage
// keeps that orientation: the MMA's M dimension walks weight rows (A operand,
// K-major, straight from the row-major weights), its N dimension walks the
// activation columns (B operand, MN-major, straight from the row-major K x N
// activations). Every stage therefore reads and writes activations in the
// reference's own K x N row-major layout, and a TMEM lane holds one output row:
// the reference's between-stage panel permutation becomes a per-thread
// shuffle of the 32 columns that thread already holds.
//
// Structure. Persistent kernel, one CTA per SM, 6 warps:
//   warp 0      TMA producer: W tile 128 x 128 B (128B swizzle) and the X tile
//               as 128-byte-wide MN-major boxes, into a STAGES-deep ring
//   warp 1      TMEM owner and MMA issuer (tcgen05.mma, one thread)
//   warps 2-5   epilogue: TMEM -> registers -> convert -> global
// Two TMEM accumulators (2 x BN columns) let the epilogue of tile t overlap
// the MMAs of tile t+1. All waits are bounded (fg_ptx.cuh).
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "fg_kernels.h"
#include "fg_ptx.cuh"

namespace fg {

constexpr int kBM = 128;          // MMA M (weight rows per tile)
constexpr int kRowBytes = 128;    // K extent of a stage in bytes (one 128B swizzle row)
constexpr int kThreads = 192;

template <int OP>
struct OpTraits;
template <>
struct OpTraits<OP_BF16> {
    static constexpr MmaKind kind = MmaKind::F16;
    static constexpr int elt = 2;
    static constexpr int BN = 256;
    static constexpr int STAGES = 4;
    static constexpr bool split = false;
    static constexpr uint32_t b_layout = SMEM_SW128;
    // D F32, A BF16, B BF16, A K-major, B MN-major
    static constexpr uint32_t idesc = make_idesc(1, 1, 1, 0, 1, kBM, BN);
};
template <>
struct OpTraits<OP_I8> {
    static constexpr MmaKind kind = MmaKind::I8;
    static constexpr int elt = 1;
    static constexpr int BN = 256;
    static constexpr int STAGES = 4;
    static constexpr bool split = false;
    static constexpr uint32_t b_layout = SMEM_SW128;
    // D S32, A U8 (the reference reads weights unsigned), B S8, A K-major, B MN-major
    static constexpr uint32_t idesc = make_idesc(2, 0, 1, 0, 1, kBM, BN);
};
template <>
struct OpTraits<OP_TF32X3> {
    static constexpr MmaKind kind = MmaKind::TF32;
    static constexpr int elt = 4;
    static constexpr int BN = 128;
    static constexpr int STAGES = 3;
    static constexpr bool split = true;
    // MN-major TF32 needs the 32-byte-chunk 128B swizzle (atoms of 4 k-rows)
    static constexpr uint32_t b_layout = SMEM_SW128_32B;
    // D F32, A TF32, B TF32, A K-major, B MN-major
    static constexpr uint32_t idesc = make_idesc(1, 2, 2, 0, 1, kBM, BN);
};

template <int OP>
struct Geometry {
    using T = OpTraits<OP>;
    static constexpr int BK = kRowBytes / T::elt;              // K elements per stage
    static constexpr int A_BYTES = kBM * kRowBytes;            // 16 KB
    static constexpr int BOX_N = kRowBytes / T::elt;           // MN-major box width (elements)
    static constexpr int BOX_BYTES = BOX_N * BK * T::elt;      // one B box
    static constexpr int NBOX = T::BN / BOX_N;
    static constexpr int B_BYTES = NBOX * BOX_BYTES;           // BN x BK elements
    static constexpr int PARTS = T::split ? 2 : 1;             // hi / lo
    static constexpr int STAGE_BYTES = PARTS * (A_BYTES + B_BYTES);
    static constexpr int MMA_K_BYTES = 32;                     // K per MMA, A side, in bytes
    static constexpr int MMAS_PER_STAGE = kRowBytes / MMA_K_BYTES;
    static constexpr int B_KSTEP_BYTES = (MMA_K_BYTES / T::elt) * kRowBytes;
    // stride between k-row groups of the B swizzle atom: 8 rows (16B chunks) or 4 rows (32B)
    static constexpr int B_SBO = T::b_layout == SMEM_SW128_32B ? 512 : 1024;
    // 3xTF32 keeps the small hi*lo + lo*hi terms in their own accumulator next to
    // hi*hi: each of the two TMEM buffers is then [hi*hi | corrections].
    static constexpr int ACC_COLS = (T::split ? 2 : 1) * T::BN;
    static constexpr int TMEM_COLS = 2 * ACC_COLS;
    static constexpr int SMEM_BYTES = T::STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*bars*/;
};

struct __align__(8) Bars {
    uint64_t full[4];
    uint64_t empty[4];
    uint64_t acc_full[2];
    uint64_t acc_empty[2];
    uint64_t mma_done;
    uint32_t tmem_base;
    int abort;
};

__device__ __forceinline__ void set_abort(Bars *b) { *reinterpret_cast<volatile int *>(&b->abort) = 1; }
__device__ __forceinline__ bool aborted(Bars *b) { return *reinterpret_cast<volatile int *>(&b->abort) != 0; }

// ------------------------------------------------------------------ epilogue helpers

__device__ __forceinline__ uint16_t f32_to_bf16_rne(float f)
{
    uint32_t u = __float_as_uint(f);
    if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40u);
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

// Round FP32 to the nearest TF32 value (10 explicit mantissa bits), ties to even.
__device__ __forceinline__ float f32_to_tf32_rne(float f)
{
    uint32_t u = __float_as_uint(f);
    if ((u & 0x7f800000u) == 0x7f800000u) return f;
    u += 0xfffu + ((u >> 13) & 1u);
    return __uint_as_float(u & 0xffffe000u);
}

__device__ __forceinline__ int8_t sat_s8(int32_t v)
{
    return (int8_t)(v > 127 ? 127 : (v < -128 ? -128 : v));
}

// Store one 32-column chunk of output row `row`, columns [n0, n0 + 32).
// v holds the raw accumulator bits (FP32 or S32).
template <int OP>
__device__ __forceinline__ void store_chunk(const StageArgs &p, int row, int n0, uint32_t (&v)[32])
{
    const int N = p.N;
    const bool full = (n0 + 32 <= N);
    // each operand kind reaches only its own epilogues; keep the others out of its code
    const int epi = OP == OP_BF16 ? (p.epi == EPI_BF16 ? EPI_BF16 : EPI_F32)
                  : OP == OP_I8   ? (p.epi == EPI_S8 ? EPI_S8 : EPI_S32)
                                  : (p.epi == EPI_TF32SPLIT ? EPI_TF32SPLIT : EPI_F32);
    switch (epi) {
    case EPI_F32:
    case EPI_S32: {
        if (row >= p.m_written) return;
        uint32_t *c = reinterpret_cast<uint32_t *>(p.out) + (size_t)row * p.ld_out + n0;
        if (full && ((p.ld_out & 3) == 0)) {
#pragma unroll
            for (int j = 0; j < 32; j += 4)
                *reinterpret_cast<uint4 *>(c + j) = make_uint4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        } else {
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (n0 + j < N) c[j] = v[j];
        }
        return;
    }
    case EPI_BF16: {
        uint16_t h[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) h[j] = f32_to_bf16_rne(__uint_as_float(v[j]));
        uint16_t *out = reinterpret_cast<uint16_t *>(p.out);
        if (p.permute && full && row < (p.M & ~1)) {
            // The reference stores the 2 x 32 block rows (2q, 2q+1) row-major and the
            // next stage reads it K-pair interleaved (multigemm/src/kernel_bf16.h:6-32,
            // :356-391): element (2q + h, c) lands at (2q + (c & 1), 16h + c / 2).
            const int hbit = row & 1;
            const int r0 = row - hbit;
            uint32_t ev[8], od[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                ev[t] = (uint32_t)h[4 * t] | ((uint32_t)h[4 * t + 2] << 16);
                od[t] = (uint32_t)h[4 * t + 1] | ((uint32_t)h[4 * t + 3] << 16);
            }
            uint16_t *d0 = out + (size_t)r0 * p.ld_out + n0 + 16 * hbit;
            uint16_t *d1 = d0 + p.ld_out;
            *reinterpret_cast<uint4 *>(d0) = make_uint4(ev[0], ev[1], ev[2], ev[3]);
            *reinterpret_cast<uint4 *>(d0 + 8) = make_uint4(ev[4], ev[5], ev[6], ev[7]);
            *reinterpret_cast<uint4 *>(d1) = make_uint4(od[0], od[1], od[2], od[3]);
            *reinterpret_cast<uint4 *>(d1 + 8) = make_uint4(od[4], od[5], od[6], od[7]);
        } else {
            uint16_t *d = out + (size_t)row * p.ld_out + n0;
            if (full && ((p.ld_out & 7) == 0)) {
                uint32_t w[16];
#pragma unroll
                for (int t = 0; t < 16; ++t) w[t] = (uint32_t)h[2 * t] | ((uint32_t)h[2 * t + 1] << 16);
#pragma unroll
                for (int t = 0; t < 16; t += 4)
                    *reinterpret_cast<uint4 *>(d + 2 * t) = make_uint4(w[t], w[t + 1], w[t + 2], w[t + 3]);
            } else {
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    if (n0 + j < N) d[j] = h[j];
            }
        }
        return;
    }
    case EPI_S8: {
        uint8_t b[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) b[j] = (uint8_t)sat_s8((int32_t)v[j]);
        uint8_t *out = reinterpret_cast<uint8_t *>(p.out);
        const int quad_rows = (p.M / 4) * 4;
        if (p.permute && full && row < quad_rows) {
            // 4 x 32 blocks: stored row-major, read K-quad interleaved
            // (multigemm/src/kernel_int8.h:6-50, :329-385): element (4q + h, c)
            // lands at (4q + (c & 3), 8h + c / 4).
            const int hq = row & 3;
            const int r0 = row - hq;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                uint32_t lo = (uint32_t)b[r] | ((uint32_t)b[r + 4] << 8) | ((uint32_t)b[r + 8] << 16) |
                              ((uint32_t)b[r + 12] << 24);
                uint32_t hi = (uint32_t)b[r + 16] | ((uint32_t)b[r + 20] << 8) |
                              ((uint32_t)b[r + 24] << 16) | ((uint32_t)b[r + 28] << 24);
                uint8_t *d = out + (size_t)(r0 + r) * p.ld_out + n0 + 8 * hq;
                *reinterpret_cast<uint2 *>(d) = make_uint2(lo, hi);
            }
        } else {
            uint8_t *d = out + (size_t)row * p.ld_out + n0;
            if (full && ((p.ld_out & 15) == 0)) {
                uint32_t w[8];
#pragma unroll
                for (int t = 0; t < 8; ++t)
                    w[t] = (uint32_t)b[4 * t] | ((uint32_t)b[4 * t + 1] << 8) |
                           ((uint32_t)b[4 * t + 2] << 16) | ((uint32_t)b[4 * t + 3] << 24);
                *reinterpret_cast<uint4 *>(d) = make_uint4(w[0], w[1], w[2], w[3]);
                *reinterpret_cast<uint4 *>(d + 16) = make_uint4(w[4], w[5], w[6], w[7]);
            } else {
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    if (n0 + j < N) d[j] = b[j];
            }
        }
        return;
    }
    case EPI_TF32SPLIT: {
        float *hi = reinterpret_cast<float *>(p.out) + (size_t)row * p.ld_out + n0;
        float *lo = reinterpret_cast<float *>(p.out_lo) + (size_t)row * p.ld_out + n0;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            if (full || n0 + j < N) {
                float x = __uint_as_float(v[j]);
                float h = f32_to_tf32_rne(x);
                hi[j] = h;
                lo[j] = f32_to_tf32_rne(x - h);
            }
        }
        return;
    }
    default:
        return;
    }
}

// ------------------------------------------------------------------ kernel

template <int OP>
__global__ void __launch_bounds__(kThreads, 1)
    tc_stage_kernel(const __grid_constant__ CUtensorMap tm_w, const __grid_constant__ CUtensorMap tm_x,
                    const __grid_constant__ CUtensorMap tm_w_lo,
                    const __grid_constant__ CUtensorMap tm_x_lo, const StageArgs p)
{
    using T = OpTraits<OP>;
    using G = Geometry<OP>;
    constexpr int BN = T::BN;
    constexpr int S = T::STAGES;

    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    Bars *bars = reinterpret_cast<Bars *>(smem + S * G::STAGE_BYTES);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int tiles_m = (p.M + kBM - 1) / kBM;
    const int tiles_n = (p.N + BN - 1) / BN;
    const int num_tiles = tiles_m * tiles_n;
    const int num_kb = (p.K + G::BK - 1) / G::BK;
    // k-blocks per accumulator hand-off. 3xTF32 hands partial sums to the
    // epilogue every p.kchunk blocks, which adds them in FP32 registers with
    // round-to-nearest: the tensor core's own FP32 accumulation over long K
    // drifts well above an FFMA loop's rounding error, short chunks do not.
    const int kchunk = (T::split && p.kchunk > 0) ? p.kchunk : num_kb;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&bars->full[s], 1);
            mbar_init(&bars->empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&bars->acc_full[a], 1);
            mbar_init(&bars->acc_empty[a], 4 * 32);
        }
        mbar_init(&bars->mma_done, 1);
        bars->abort = 0;
        fence_mbar_init();
    }
    if (warp == 0 && lane == 0) {
        tma_prefetch_desc(&tm_w);
        tma_prefetch_desc(&tm_x);
        if constexpr (T::split) {
            tma_prefetch_desc(&tm_w_lo);
            tma_prefetch_desc(&tm_x_lo);
        }
    }
    if (warp == 1) tmem_alloc(&bars->tmem_base, G::TMEM_COLS);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = bars->tmem_base;

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            uint32_t pending = 0;      // bit s: stage s has loads issued
            uint32_t pending_ph = 0;   // bit s: parity of stage s's last issue
            for (int t = blockIdx.x; t < num_tiles; t += gridDim.x) {
                const int m0 = (t / tiles_n) * kBM;
                const int n0 = (t % tiles_n) * BN;
                // boxes that start past the last column are skipped: their columns
                // only feed output columns that are never stored
                int nvb = (p.N - n0 + G::BOX_N - 1) / G::BOX_N;
                nvb = nvb < G::NBOX ? nvb : G::NBOX;
                const uint32_t tx_bytes = G::PARTS * (G::A_BYTES + nvb * G::BOX_BYTES);
                for (int kb = 0; kb < num_kb; ++kb) {
                    if (!mbar_wait(&bars->empty[s], ph ^ 1, p.status, KERR_WAIT_EMPTY)) {
                        set_abort(bars);
                        goto producer_done;
                    }
                    uint8_t *st = smem + s * G::STAGE_BYTES;
                    mbar_arrive_expect_tx(&bars->full[s], tx_bytes);
                    const int k0 = kb * G::BK;
                    tma_load_2d(st, &tm_w, &bars->full[s], k0, m0);
                    for (int j = 0; j < nvb; ++j)
                        tma_load_2d(st + G::A_BYTES + j * G::BOX_BYTES, &tm_x, &bars->full[s],
                                    n0 + j * G::BOX_N, k0);
                    if constexpr (T::split) {
                        uint8_t *st2 = st + G::A_BYTES + G::B_BYTES;
                        tma_load_2d(st2, &tm_w_lo, &bars->full[s], k0, m0);
                        for (int j = 0; j < nvb; ++j)
                            tma_load_2d(st2 + G::A_BYTES + j * G::BOX_BYTES, &tm_x_lo,
                                        &bars->full[s], n0 + j * G::BOX_N, k0);
                    }
                    pending |= 1u << s;
                    pending_ph = (pending_ph & ~(1u << s)) | (ph << s);
                    if (++s == S) {
                        s = 0;
                        ph ^= 1;
                    }
                }
                if (aborted(bars)) break;
            }
        producer_done:
            // never leave with copies in flight into this CTA's shared memory
            for (int st = 0; st < S; ++st)
                if (pending & (1u << st))
                    mbar_wait(&bars->full[st], (pending_ph >> st) & 1u, p.status, KERR_WAIT_FULL);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            int acc = 0;
            uint32_t acc_ph = 0;
            for (int t = blockIdx.x; t < num_tiles; t += gridDim.x) {
                // one accumulator hand-off per chunk of k-blocks (the whole K unless
                // the epilogue promotes partial sums, see kchunk)
                for (int kc = 0; kc < num_kb; kc += kchunk) {
                    if (!mbar_wait(&bars->acc_empty[acc], acc_ph ^ 1, p.status,
                                   KERR_WAIT_ACC_EMPTY)) {
                        set_abort(bars);
                        goto mma_done;
                    }
                    tc_fence_after();
                    const uint32_t d_tmem = tmem_base + acc * G::ACC_COLS;
                    const int kend = kc + kchunk < num_kb ? kc + kchunk : num_kb;
                    for (int kb = kc; kb < kend; ++kb) {
                        if (!mbar_wait(&bars->full[s], ph, p.status, KERR_WAIT_FULL)) {
                            set_abort(bars);
                            goto mma_done;
                        }
                        tc_fence_after();
                        const uint32_t a_addr = smem_u32(smem + s * G::STAGE_BYTES);
                        const uint32_t b_addr = a_addr + G::A_BYTES;
#pragma unroll
                        for (int k = 0; k < G::MMAS_PER_STAGE; ++k) {
                            const uint64_t ad =
                                smem_desc(a_addr + k * G::MMA_K_BYTES, 16, 1024, SMEM_SW128);
                            const uint64_t bd = smem_desc(b_addr + k * G::B_KSTEP_BYTES,
                                                          G::BOX_BYTES, G::B_SBO, T::b_layout);
                            const uint32_t accumulate = (kb != kc || k != 0);
                            if constexpr (T::split) {
                                const uint32_t lo_off = G::A_BYTES + G::B_BYTES;
                                const uint64_t ad_lo = smem_desc(
                                    a_addr + lo_off + k * G::MMA_K_BYTES, 16, 1024, SMEM_SW128);
                                const uint64_t bd_lo =
                                    smem_desc(b_addr + lo_off + k * G::B_KSTEP_BYTES,
                                              G::BOX_BYTES, G::B_SBO, T::b_layout);
                                // hi*lo + lo*hi into the correction accumulator, whose
                                // rounding is 2^-11 smaller; hi*hi alone into the main one
                                tc_mma<T::kind>(d_tmem + BN, ad, bd_lo, T::idesc, accumulate);
                                tc_mma<T::kind>(d_tmem + BN, ad_lo, bd, T::idesc, 1);
                                tc_mma<T::kind>(d_tmem, ad, bd, T::idesc, accumulate);
                            } else {
                                tc_mma<T::kind>(d_tmem, ad, bd, T::idesc, accumulate);
                            }
                        }
                        tc_commit(&bars->empty[s]);  // stage free once these MMAs retire
                        if (++s == S) {
                            s = 0;
                            ph ^= 1;
                        }
                    }
                    tc_commit(&bars->acc_full[acc]);  // accumulator ready once its MMAs retire
                    if (++acc == 2) {
                        acc = 0;
                        acc_ph ^= 1;
                    }
                }
                if (aborted(bars)) break;
            }
        mma_done:
            // all MMAs this thread issued have retired before TMEM is released
            tc_commit(&bars->mma_done);
            mbar_wait(&bars->mma_done, 0, p.status, KERR_WAIT_FULL);
        }
    } else {
        // ------------------------------------------------------------ epilogue (warps 2..5)
        const int quarter = warp & 3;  // TMEM lane quarter this warp may access
        int acc = 0;
        uint32_t acc_ph = 0;
        if constexpr (T::split) {
            for (int t = blockIdx.x; t < num_tiles; t += gridDim.x) {
                const int m0 = (t / tiles_n) * kBM;
                const int n0 = (t % tiles_n) * BN;
                const int row = m0 + quarter * 32 + lane;
                float sum[BN / 32][32];
#pragma unroll
                for (int c = 0; c < BN / 32; ++c)
#pragma unroll
                    for (int j = 0; j < 32; ++j) sum[c][j] = 0.f;
                bool ok = true;
                for (int kc = 0; kc < num_kb; kc += kchunk) {
                    if (!mbar_wait(&bars->acc_full[acc], acc_ph, p.status, KERR_WAIT_ACC_FULL)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t t_row =
                        tmem_base + acc * G::ACC_COLS + ((uint32_t)(quarter * 32) << 16);
#pragma unroll
                    for (int c = 0; c < BN / 32; ++c) {
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            uint32_t v[16], w[16];
                            tmem_ld_32x32b_x16(t_row + c * 32 + 16 * h, v);
                            tmem_ld_32x32b_x16(t_row + BN + c * 32 + 16 * h, w);
                            tmem_ld_wait();
#pragma unroll
                            for (int j = 0; j < 16; ++j)
                                sum[c][16 * h + j] = sum[c][16 * h + j] +
                                                     (__uint_as_float(v[j]) + __uint_as_float(w[j]));
                        }
                    }
                    tc_fence_before();
                    mbar_arrive(&bars->acc_empty[acc]);
                    if (++acc == 2) {
                        acc = 0;
                        acc_ph ^= 1;
                    }
                }
                if (!ok) {
                    set_abort(bars);
                    break;
                }
#pragma unroll
                for (int c = 0; c < BN / 32; ++c) {
                    const int nc = n0 + c * 32;
                    if (nc < p.N && row < p.M) {
                        uint32_t v[32];
#pragma unroll
                        for (int j = 0; j < 32; ++j) v[j] = __float_as_uint(sum[c][j]);
                        store_chunk<OP>(p, row, nc, v);
                    }
                }
                if (aborted(bars)) break;
            }
        } else
        for (int t = blockIdx.x; t < num_tiles; t += gridDim.x) {
            if (!mbar_wait(&bars->acc_full[acc], acc_ph, p.status, KERR_WAIT_ACC_FULL)) {
                set_abort(bars);
                break;
            }
            tc_fence_after();
            const int m0 = (t / tiles_n) * kBM;
            const int n0 = (t % tiles_n) * BN;
            const int row = m0 + quarter * 32 + lane;
            const uint32_t t_row = tmem_base + acc * G::ACC_COLS + ((uint32_t)(quarter * 32) << 16);
            const bool tail = (row >= p.tail_lo && row < p.tail_hi);
            uint32_t wq = 0;
            if (tail) wq = *reinterpret_cast<const uint32_t *>(
                              reinterpret_cast<const uint8_t *>(p.w) + (size_t)row * p.ld_w + p.K);
#pragma unroll 1
            for (int c = 0; c < BN / 32; ++c) {
                uint32_t v[32];
                tmem_ld_32x32b_x32(t_row + c * 32, v);
                tmem_ld_wait();
                const int nc = n0 + c * 32;
                if (nc >= p.N) continue;  // whole chunk past the last column (warp-uniform)
                if (tail) {
                    // INT8 reference tail rows: add back weight quad 0 * activation quad 0
                    const int8_t *x = reinterpret_cast<const int8_t *>(p.x);
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        const int a = (int)((wq >> (8 * r)) & 0xffu);
                        const int8_t *xr = x + (size_t)r * p.ld_x + nc;
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (nc + j < p.N) v[j] = (uint32_t)((int32_t)v[j] + a * (int32_t)xr[j]);
                    }
                }
                if (row < p.M) store_chunk<OP>(p, row, nc, v);
            }
            tc_fence_before();
            mbar_arrive(&bars->acc_empty[acc]);
            if (++acc == 2) {
                acc = 0;
                acc_ph ^= 1;
            }
            if (aborted(bars)) break;
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem_base, G::TMEM_COLS);
    }
}

// ------------------------------------------------------------------ host side

using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                   const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                   const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// Row-major rows x cols matrix with leading dimension ld (elements); box is
// box_cols (innermost, 128 bytes) x box_rows, 128-byte swizzle, zero fill.
static bool make_map(CUtensorMap *m, CUtensorMapDataType dt, int elt, const void *base, long rows,
                     long cols, long ld, int box_cols, int box_rows,
                     CUtensorMapSwizzle swz = CU_TENSOR_MAP_SWIZZLE_128B)
{
    EncodeTiledFn enc = encode_fn();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * elt};
    cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, dt, 2, const_cast<void *>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, swz,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

template <int OP>
static cudaError_t launch_op(const StageArgs &a, int num_sms, cudaStream_t s)
{
    using T = OpTraits<OP>;
    using G = Geometry<OP>;
    CUtensorMapDataType dt = OP == OP_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                             : OP == OP_I8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                           : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const CUtensorMapSwizzle bswz = T::b_layout == SMEM_SW128_32B
                                        ? CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B
                                        : CU_TENSOR_MAP_SWIZZLE_128B;
    CUtensorMap tw, tx, twl, txl;
    if (!make_map(&tw, dt, T::elt, a.w, a.M, a.K, a.ld_w, G::BK, kBM)) return cudaErrorInvalidValue;
    if (!make_map(&tx, dt, T::elt, a.x, a.K, a.N, a.ld_x, G::BOX_N, G::BK, bswz))
        return cudaErrorInvalidValue;
    if (T::split) {
        if (!make_map(&twl, dt, T::elt, a.w_lo, a.M, a.K, a.ld_w, G::BK, kBM)) return cudaErrorInvalidValue;
        if (!make_map(&txl, dt, T::elt, a.x_lo, a.K, a.N, a.ld_x, G::BOX_N, G::BK, bswz))
            return cudaErrorInvalidValue;
    } else {
        twl = tw;
        txl = tx;
    }
    static unsigned long long attr_set = 0;  // bit per device: the attribute is per context
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(attr_set & (1ull << (dev & 63)))) {
        cudaError_t e = cudaFuncSetAttribute(tc_stage_kernel<OP>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        attr_set |= 1ull << (dev & 63);
    }
    const int tiles = ((a.M + kBM - 1) / kBM) * ((a.N + T::BN - 1) / T::BN);
    const int grid = tiles < num_sms ? tiles : num_sms;
    tc_stage_kernel<OP><<<grid, kThreads, G::SMEM_BYTES, s>>>(tw, tx, twl, txl, a);
    return cudaGetLastError();
}

cudaError_t launch_tc_stage(const StageArgs &a, int num_sms, cudaStream_t s)
{
    if (a.M <= 0 || a.N <= 0 || a.K <= 0) return cudaErrorInvalidValue;
    switch (a.op) {
    case OP_BF16: return launch_op<OP_BF16>(a, num_sms, s);
    case OP_I8: return launch_op<OP_I8>(a, num_sms, s);
    case OP_TF32X3: return launch_op<OP_TF32X3>(a, num_sms, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace fg
