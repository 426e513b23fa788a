// Pieces shared by the tensor-core kernels (fg_gemm_tc.cu: one GEMM stage per
// launch; fg_chain_fused.cu: a whole chain per launch): tile geometry, the
// shared-memory barrier block, the epilogue (TMEM -> registers -> the stage's
// output format, including the reference's panel permutation) and the TMA
// tensor-map encoding on the host.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
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
    // Two accumulators of BN columns. 3xTF32 keeps the small hi*lo + lo*hi terms
    // in their own accumulators at CORR_COLS (one per tile in flight), summed over
    // the whole tile, while hi*hi is handed to the epilogue chunk by chunk.
    static constexpr int ACC_COLS = T::BN;
    static constexpr int CORR_COLS = 2 * T::BN;
    static constexpr int TMEM_COLS = (T::split ? 4 : 2) * T::BN;
    static constexpr int STAGING_BYTES = 4 * 2 * 4096;  // TMA-store epilogue, 2 buffers per warp
    static constexpr int SMEM_BYTES =
        T::STAGES * STAGE_BYTES + STAGING_BYTES + 1024 /*align*/ + 256 /*bars*/;
};

struct __align__(8) Bars {
    uint64_t full[8];
    uint64_t empty[8];
    uint64_t acc_full[2];
    uint64_t acc_empty[2];
    uint64_t mma_done;
    uint32_t tmem_base;
    int abort;
};

__device__ __forceinline__ void set_abort(Bars *b) { *reinterpret_cast<volatile int *>(&b->abort) = 1; }
__device__ __forceinline__ bool aborted(Bars *b) { return *reinterpret_cast<volatile int *>(&b->abort) != 0; }

// Whether the 128 weight rows starting at m0 hold INT8 tail rows, which are
// then loaded from the pre-shifted tail block instead of the weights.
__device__ __forceinline__ bool tile_has_tail(const StageArgs &p, int m0)
{
    return p.tail_hi > p.tail_lo && m0 < p.tail_hi && m0 + 128 > p.tail_lo;
}

// ------------------------------------------------------------------ epilogue helpers

__device__ __forceinline__ uint16_t f32_to_bf16_rne(float f)
{
    uint32_t u = __float_as_uint(f);
    if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40u);
    u += 0x7fffu + ((u >> 16) & 1u);
    return (uint16_t)(u >> 16);
}

// Round FP32 to the nearest TF32 value (10 explicit mantissa bits), ties to
// even, as an FP32 bit pattern with the low 13 bits clear: one cvt.rn.tf32.f32.
// For every finite input this equals rounding the low 13 bits of the pattern
// as an integer (add 0xfff plus bit 13, clear the low bits); that was checked
// on B200 over all 2^32 patterns.
__device__ __forceinline__ float f32_to_tf32_rne(float f)
{
    uint32_t r;
    asm("cvt.rn.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
    return __uint_as_float(r);
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

// Read one finished accumulator tile row (TMEM lane = output row `row`,
// columns n0 .. n0 + BN) and store it through the stage's epilogue.
template <int OP, int BN>
__device__ __noinline__ void drain_tile(const StageArgs &p, uint32_t t_row, int row, int n0)
{
    const bool tail = (row >= p.tail_lo && row < p.tail_hi);
    uint32_t wq = 0;
    if (tail)
        wq = *reinterpret_cast<const uint32_t *>(reinterpret_cast<const uint8_t *>(p.w_tail) +
                                                 (size_t)(row - p.tail_row0) * p.ld_w_tail + p.K);
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
}

// ------------------------------------------------------------------ staged (TMA-store) epilogue
//
// Each epilogue warp owns 32 output rows of a tile (its TMEM lane quarter) and
// two 4 KB staging buffers of 32 rows x 128 bytes in shared memory, 128-byte
// swizzled (16-byte chunk j of row r at chunk j ^ (r % 8): conflict-free for
// the row-per-lane writes below). A buffer holds 32 FP32/int32 columns, 64
// BF16 columns or 128 int8 columns; once written it goes out as one TMA bulk
// store (coalesced, asynchronous, clipped at the tensor's edges) while the
// warp fills the other buffer.

constexpr int kStageBufBytes = 4096;
constexpr int kEpiStagingBytes = 4 * 2 * kStageBufBytes;  // 4 warps x 2 buffers

__device__ __forceinline__ void st_sw16(uint8_t *sb, int r, int byte_off, uint4 v)
{
    const int chunk = (byte_off >> 4) ^ (r & 7);
    *reinterpret_cast<uint4 *>(sb + r * 128 + chunk * 16) = v;
}

__device__ __forceinline__ void st_sw8(uint8_t *sb, int r, int byte_off, uint2 v)
{
    const int chunk = (byte_off >> 4) ^ (r & 7);
    *reinterpret_cast<uint2 *>(sb + r * 128 + chunk * 16 + (byte_off & 8)) = v;
}

// Two FP32 values to packed BF16 (a in the low half), round to nearest even:
// one cvt.rn.bf16x2.f32.
__device__ __forceinline__ uint32_t pack_bf16x2(uint32_t a, uint32_t b)
{
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(__uint_as_float(b)), "f"(__uint_as_float(a)));
    return r;
}

// Four int32 to packed saturated int8 (a in the low byte): two
// cvt.pack.sat.s8.s32.b32, each of which saturates two values into the low 16
// bits of its result and copies the low 16 bits of its third operand above them.
__device__ __forceinline__ uint32_t pack_s8x4(uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
    uint32_t hi, r;
    asm("cvt.pack.sat.s8.s32.b32 %0, %1, %2, %3;" : "=r"(hi) : "r"(d), "r"(c), "r"(0u));
    asm("cvt.pack.sat.s8.s32.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(b), "r"(a), "r"(hi));
    return r;
}

// Write TMEM chunk `cc` (32 columns, this lane's row r) of a staging buffer.
// col_in_buf: first column of the chunk inside the buffer; full: the chunk's 32
// columns are a whole panel inside N (only then is the permutation applied).
template <int EPI>
__device__ __forceinline__ void stage_chunk(const StageArgs &p, uint8_t *sb, int r, int row,
                                            int col_in_buf, bool full, const uint32_t (&v)[32])
{
    if constexpr (EPI == EPI_F32 || EPI == EPI_S32) {
#pragma unroll
        for (int j = 0; j < 8; ++j)
            st_sw16(sb, r, col_in_buf * 4 + 16 * j,
                    make_uint4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]));
    } else if constexpr (EPI == EPI_BF16) {
        const int base = col_in_buf * 2;  // bytes
        if (p.permute && full && row < (p.M & ~1)) {
            // element (2q + h, c) of the 2 x 32 block goes to (2q + (c & 1), 16h + c / 2)
            // (multigemm/src/kernel_bf16.h:6-32 read of the :356-391 row-major store)
            const int h = r & 1;
            const int r0 = r - h;
            uint32_t e[8], o[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                e[t] = pack_bf16x2(v[4 * t], v[4 * t + 2]);
                o[t] = pack_bf16x2(v[4 * t + 1], v[4 * t + 3]);
            }
            st_sw16(sb, r0, base + 32 * h, make_uint4(e[0], e[1], e[2], e[3]));
            st_sw16(sb, r0, base + 32 * h + 16, make_uint4(e[4], e[5], e[6], e[7]));
            st_sw16(sb, r0 + 1, base + 32 * h, make_uint4(o[0], o[1], o[2], o[3]));
            st_sw16(sb, r0 + 1, base + 32 * h + 16, make_uint4(o[4], o[5], o[6], o[7]));
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                st_sw16(sb, r, base + 16 * j,
                        make_uint4(pack_bf16x2(v[8 * j], v[8 * j + 1]),
                                   pack_bf16x2(v[8 * j + 2], v[8 * j + 3]),
                                   pack_bf16x2(v[8 * j + 4], v[8 * j + 5]),
                                   pack_bf16x2(v[8 * j + 6], v[8 * j + 7])));
        }
    } else {  // EPI_S8
        const int base = col_in_buf;  // bytes
        if (p.permute && full && row < (p.M / 4) * 4) {
            // element (4q + h, c) of the 4 x 32 block goes to (4q + (c & 3), 8h + c / 4)
            // (multigemm/src/kernel_int8.h:6-50 read of the :329-385 row-major store)
            const int hq = r & 3;
            const int r0 = r - hq;
#pragma unroll
            for (int rr = 0; rr < 4; ++rr)
                st_sw8(sb, r0 + rr, base + 8 * hq,
                       make_uint2(pack_s8x4(v[rr], v[rr + 4], v[rr + 8], v[rr + 12]),
                                  pack_s8x4(v[rr + 16], v[rr + 20], v[rr + 24], v[rr + 28])));
        } else {
#pragma unroll
            for (int j = 0; j < 2; ++j)
                st_sw16(sb, r, base + 16 * j,
                        make_uint4(pack_s8x4(v[16 * j], v[16 * j + 1], v[16 * j + 2], v[16 * j + 3]),
                                   pack_s8x4(v[16 * j + 4], v[16 * j + 5], v[16 * j + 6], v[16 * j + 7]),
                                   pack_s8x4(v[16 * j + 8], v[16 * j + 9], v[16 * j + 10], v[16 * j + 11]),
                                   pack_s8x4(v[16 * j + 12], v[16 * j + 13], v[16 * j + 14],
                                             v[16 * j + 15])));
        }
    }
}

// INT8 reference tail rows: add back weight quad 0 x activation quad 0. The
// whole warp takes part (it loads each column's input quad once, lane l column
// nc + l, and passes it round); lanes of tail rows add it with one mixed-sign
// dp4a (weight bytes unsigned, input bytes signed), exact in int32.
__device__ __forceinline__ void tail_fix(const StageArgs &p, uint32_t wq, bool tail, int nc, int lane,
                                         uint32_t (&v)[32])
{
    const uint8_t *x = reinterpret_cast<const uint8_t *>(p.x);
    uint32_t qp = 0;
    if (nc + lane < p.N)
#pragma unroll
        for (int q = 0; q < 4; ++q) qp |= (uint32_t)x[(size_t)q * p.ld_x + nc + lane] << (8 * q);
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        const uint32_t qj = __shfl_sync(0xffffffffu, qp, j);
        if (tail && nc + j < p.N) {
            int r;
            asm("dp4a.u32.s32 %0, %1, %2, %3;" : "=r"(r) : "r"(wq), "r"(qj), "r"((int)v[j]));
            v[j] = (uint32_t)r;
        }
    }
}

template <int OP, int BN, int EPI>
__device__ __forceinline__ void drain_staged(const StageArgs &p, const CUtensorMap *tm_out,
                                             uint32_t t_row, int lane, int warp_row0, int n0,
                                             uint8_t *staging, int &sbuf)
{
    constexpr int COLS = (EPI == EPI_BF16) ? 64 : (EPI == EPI_S8) ? 128 : 32;  // per buffer
    constexpr int CPB = COLS / 32;                                             // chunks per buffer
    const int row = warp_row0 + lane;
    const bool tail = (row >= p.tail_lo && row < p.tail_hi);
    uint32_t wq = 0;
    if (tail)
        wq = *reinterpret_cast<const uint32_t *>(reinterpret_cast<const uint8_t *>(p.w_tail) +
                                                 (size_t)(row - p.tail_row0) * p.ld_w_tail + p.K);
    const bool rows_in = warp_row0 < p.M;
    const bool warp_tail = __any_sync(0xffffffffu, tail);
#pragma unroll 1
    for (int b = 0; b < BN / COLS; ++b) {
        const int col0 = n0 + b * COLS;
        if (col0 >= p.N) break;  // warp-uniform
        uint8_t *sb = staging + sbuf * kStageBufBytes;
        if (lane == 0) bulk_wait_read<1>();  // this buffer's previous store has read it
        __syncwarp();
#pragma unroll
        for (int cc = 0; cc < CPB; cc += 2) {
            uint32_t va[32], vb[32];
            tmem_ld_32x32b_x32(t_row + (b * CPB + cc) * 32, va);
            if (CPB > 1) tmem_ld_32x32b_x32(t_row + (b * CPB + cc + 1) * 32, vb);
            tmem_ld_wait();
            const int nca = col0 + cc * 32;
            if (warp_tail) tail_fix(p, wq, tail, nca, lane, va);
            stage_chunk<EPI>(p, sb, lane, row, cc * 32, nca + 32 <= p.N, va);
            if (CPB > 1) {
                const int ncb = nca + 32;
                if (warp_tail) tail_fix(p, wq, tail, ncb, lane, vb);
                stage_chunk<EPI>(p, sb, lane, row, (cc + 1) * 32, ncb + 32 <= p.N, vb);
            }
        }
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0 && rows_in) {
            // a chain's result is not read again in the launch: first out of L2, so
            // that the intermediates the next stages read stay in it
            if constexpr (EPI == EPI_BF16 || EPI == EPI_S8) {
                // an intermediate: kept in L2 where asked, so that the later stage
                // that overwrites the buffer finds it there and it is never written back
                if (p.l2_keep)
                    tma_store_2d_hint(tm_out, sb, col0, warp_row0, l2_policy_evict_last());
                else
                    tma_store_2d(tm_out, sb, col0, warp_row0);
            } else
                tma_store_2d_hint(tm_out, sb, col0, warp_row0, l2_policy_evict_first());
            bulk_commit();
        }
        sbuf ^= 1;
    }
}

// Epilogue of one tile row block for one warp: TMA-staged when the launcher
// could map the output, else direct stores.
template <int OP, int BN>
__device__ __forceinline__ void drain_warp(const StageArgs &p, const CUtensorMap *tm_out,
                                           uint32_t t_row, int lane, int warp_row0, int n0,
                                           uint8_t *staging, int &sbuf)
{
    if (p.tma_store) {
        if constexpr (OP == OP_BF16) {
            if (p.epi == EPI_BF16)
                drain_staged<OP, BN, EPI_BF16>(p, tm_out, t_row, lane, warp_row0, n0, staging, sbuf);
            else
                drain_staged<OP, BN, EPI_F32>(p, tm_out, t_row, lane, warp_row0, n0, staging, sbuf);
        } else if constexpr (OP == OP_I8) {
            if (p.epi == EPI_S8)
                drain_staged<OP, BN, EPI_S8>(p, tm_out, t_row, lane, warp_row0, n0, staging, sbuf);
            else
                drain_staged<OP, BN, EPI_S32>(p, tm_out, t_row, lane, warp_row0, n0, staging, sbuf);
        }
    } else {
        drain_tile<OP, BN>(p, t_row, warp_row0 + lane, n0);
    }
}

template <int OP>
struct PairGeo {
    using T = OpTraits<OP>;
    static constexpr int BM = 256;                                // pair tile rows
    static constexpr int BN = 256;                                // pair tile columns
    static constexpr int BK = kRowBytes / T::elt;
    static constexpr int A_BYTES = 128 * kRowBytes;               // this CTA's 128 rows
    static constexpr int BOX_N = kRowBytes / T::elt;
    static constexpr int BOX_BYTES = BOX_N * BK * T::elt;
    static constexpr int NBOX = (BN / 2) / BOX_N;                 // this CTA's 128 columns
    static constexpr int B_BYTES = NBOX * BOX_BYTES;
    static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;         // 32 KB
    static constexpr int STAGES = 6;
    static constexpr int MMA_K_BYTES = 32;
    static constexpr int MMAS_PER_STAGE = kRowBytes / MMA_K_BYTES;
    static constexpr int B_KSTEP_BYTES = (MMA_K_BYTES / T::elt) * kRowBytes;
    static constexpr int TMEM_COLS = 2 * BN;                      // two accumulators
    static constexpr int STAGING_BYTES = kEpiStagingBytes;
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + STAGING_BYTES + 1024 + 256;
    static constexpr uint32_t idesc = OP == OP_BF16 ? make_idesc(1, 1, 1, 0, 1, BM, BN)
                                                    : make_idesc(2, 0, 1, 0, 1, BM, BN);
};


// ------------------------------------------------------------------ host side

using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                   const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                   const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_fn()
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
inline bool make_map(CUtensorMap *m, CUtensorMapDataType dt, int elt, const void *base, long rows,
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


// Tensor map for a stage's output and whether TMA bulk stores can write it
// (16-byte-aligned base and rows); box = one staging buffer (32 rows x 128 B).
inline bool make_out_map(CUtensorMap *m, const StageArgs &a)
{
    CUtensorMapDataType dt;
    int elt, box_cols;
    long rows = a.M;
    switch (a.epi) {
    case EPI_F32: dt = CU_TENSOR_MAP_DATA_TYPE_FLOAT32; elt = 4; box_cols = 32; break;
    case EPI_S32: dt = CU_TENSOR_MAP_DATA_TYPE_INT32; elt = 4; box_cols = 32; rows = a.m_written; break;
    case EPI_BF16: dt = CU_TENSOR_MAP_DATA_TYPE_BFLOAT16; elt = 2; box_cols = 64; break;
    case EPI_S8: dt = CU_TENSOR_MAP_DATA_TYPE_UINT8; elt = 1; box_cols = 128; break;
    default: return false;
    }
    if (rows <= 0 || ((uintptr_t)a.out & 15) || ((a.ld_out * elt) & 15)) return false;
    return make_map(m, dt, elt, a.out, rows, a.N, a.ld_out, box_cols, 32);
}

}  // namespace fg
