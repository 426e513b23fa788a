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

#include <mutex>

#include <cstdio>
#include <cstdlib>

#include "fg_tc_common.cuh"

namespace fg {

// ------------------------------------------------------------------ kernel

template <int OP>
__global__ void __launch_bounds__(kThreads, 1)
    tc_stage_kernel(const __grid_constant__ CUtensorMap tm_w, const __grid_constant__ CUtensorMap tm_x,
                    const __grid_constant__ CUtensorMap tm_w_lo,
                    const __grid_constant__ CUtensorMap tm_x_lo,
                    const __grid_constant__ CUtensorMap tm_out,
                    const __grid_constant__ CUtensorMap tm_out2, const StageArgs p)
{
    using T = OpTraits<OP>;
    using G = Geometry<OP>;
    constexpr int BN = T::BN;
    constexpr int S = T::STAGES;

    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    Bars *bars = reinterpret_cast<Bars *>(smem + S * G::STAGE_BYTES + G::STAGING_BYTES);

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
        if constexpr (T::split)
            for (int a = 0; a < 2; ++a) {
                mbar_init(&bars->full[6 + a], 1);        // correction ready
                mbar_init(&bars->empty[6 + a], 4 * 32);  // correction drained
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
                    if (OP == OP_I8 && tile_has_tail(p, m0))  // INT8: tail block in tm_w_lo
                        tma_load_2d(st, &tm_w_lo, &bars->full[s], k0, m0 - p.tail_row0);
                    else
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
            int cb = 0;  // 3xTF32: correction accumulator of this tile
            uint32_t cb_ph = 0;
            for (int t = blockIdx.x; t < num_tiles; t += gridDim.x) {
                uint32_t c_tmem = 0;
                if constexpr (T::split) {
                    if (!mbar_wait(&bars->empty[6 + cb], cb_ph ^ 1, p.status, KERR_WAIT_ACC_EMPTY)) {
                        set_abort(bars);
                        goto mma_done;
                    }
                    tc_fence_after();
                    c_tmem = tmem_base + G::CORR_COLS + cb * T::BN;
                }
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
                                // hi*lo + lo*hi into the tile's correction accumulator,
                                // whose rounding is 2^-11 smaller; hi*hi alone into the
                                // chunk's main one
                                tc_mma<T::kind>(c_tmem, ad, bd_lo, T::idesc, (kb | k) != 0);
                                tc_mma<T::kind>(c_tmem, ad_lo, bd, T::idesc, 1);
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
                if constexpr (T::split) {
                    tc_commit(&bars->full[6 + cb]);
                    if (++cb == 2) {
                        cb = 0;
                        cb_ph ^= 1;
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
            int cb = 0;
            uint32_t cb_ph = 0;
            uint8_t *staging = smem + S * G::STAGE_BYTES + (warp - 2) * 2 * kStageBufBytes;
            int sbuf = 0;
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
                        uint32_t v[32];
                        tmem_ld_32x32b_x32(t_row + c * 32, v);
                        tmem_ld_wait();
#pragma unroll
                        for (int j = 0; j < 32; ++j) sum[c][j] = sum[c][j] + __uint_as_float(v[j]);
                    }
                    tc_fence_before();
                    mbar_arrive(&bars->acc_empty[acc]);
                    if (++acc == 2) {
                        acc = 0;
                        acc_ph ^= 1;
                    }
                }
                // the tile's correction terms, added once
                if (ok && !mbar_wait(&bars->full[6 + cb], cb_ph, p.status, KERR_WAIT_ACC_FULL))
                    ok = false;
                if (ok) {
                    tc_fence_after();
                    const uint32_t t_row = tmem_base + G::CORR_COLS + cb * BN +
                                           ((uint32_t)(quarter * 32) << 16);
#pragma unroll
                    for (int c = 0; c < BN / 32; ++c) {
                        uint32_t w[32];
                        tmem_ld_32x32b_x32(t_row + c * 32, w);
                        tmem_ld_wait();
#pragma unroll
                        for (int j = 0; j < 32; ++j) sum[c][j] = sum[c][j] + __uint_as_float(w[j]);
                    }
                    tc_fence_before();
                    mbar_arrive(&bars->empty[6 + cb]);
                    if (++cb == 2) {
                        cb = 0;
                        cb_ph ^= 1;
                    }
                }
                if (!ok) {
                    set_abort(bars);
                    break;
                }
                if (p.tma_store) {
                    // staged TMA stores, 32 columns at a time: the FP32 result, or the
                    // (hi, lo) TF32 pair of the next stage's input in the two buffers
                    const int warp_row0 = m0 + quarter * 32;
                    const bool rows_in = warp_row0 < p.M;
                    const bool split_out = p.epi == EPI_TF32SPLIT;
#pragma unroll
                    for (int c = 0; c < BN / 32; ++c) {
                        const int nc = n0 + c * 32;
                        if (nc >= p.N) break;  // warp-uniform
                        uint8_t *b0 = staging + (split_out ? 0 : sbuf) * kStageBufBytes;
                        uint8_t *b1 = staging + kStageBufBytes;
                        if (lane == 0) {
                            if (split_out)
                                bulk_wait_read<0>();
                            else
                                bulk_wait_read<1>();
                        }
                        __syncwarp();
                        if (split_out) {
#pragma unroll
                            for (int j = 0; j < 8; ++j) {
                                uint32_t h[4], l[4];
#pragma unroll
                                for (int u = 0; u < 4; ++u) {
                                    const float x = sum[c][4 * j + u];
                                    const float hf = f32_to_tf32_rne(x);
                                    h[u] = __float_as_uint(hf);
                                    l[u] = __float_as_uint(f32_to_tf32_rne(x - hf));
                                }
                                st_sw16(b0, lane, 16 * j, make_uint4(h[0], h[1], h[2], h[3]));
                                st_sw16(b1, lane, 16 * j, make_uint4(l[0], l[1], l[2], l[3]));
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < 8; ++j)
                                st_sw16(b0, lane, 16 * j,
                                        make_uint4(__float_as_uint(sum[c][4 * j]),
                                                   __float_as_uint(sum[c][4 * j + 1]),
                                                   __float_as_uint(sum[c][4 * j + 2]),
                                                   __float_as_uint(sum[c][4 * j + 3])));
                            sbuf ^= 1;
                        }
                        fence_proxy_async_smem();
                        __syncwarp();
                        if (lane == 0 && rows_in) {
                            tma_store_2d(&tm_out, b0, nc, warp_row0);
                            if (split_out) tma_store_2d(&tm_out2, b1, nc, warp_row0);
                            bulk_commit();
                        }
                    }
                } else {
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
                }
                if (aborted(bars)) break;
            }
        } else {
        uint8_t *staging = smem + S * G::STAGE_BYTES + (warp - 2) * 2 * kStageBufBytes;
        int sbuf = 0;
        for (int t = blockIdx.x; t < num_tiles; t += gridDim.x) {
            if (!mbar_wait(&bars->acc_full[acc], acc_ph, p.status, KERR_WAIT_ACC_FULL)) {
                set_abort(bars);
                break;
            }
            tc_fence_after();
            const int m0 = (t / tiles_n) * kBM;
            const int n0 = (t % tiles_n) * BN;
            const uint32_t t_row = tmem_base + acc * G::ACC_COLS + ((uint32_t)(quarter * 32) << 16);
            drain_warp<OP, BN>(p, &tm_out, t_row, lane, m0 + quarter * 32, n0, staging, sbuf);
            tc_fence_before();
            mbar_arrive(&bars->acc_empty[acc]);
            if (++acc == 2) {
                acc = 0;
                acc_ph ^= 1;
            }
            if (aborted(bars)) break;
        }
        }
    }

    if (warp >= 2 && lane == 0) bulk_wait<0>();  // staged stores done before shared memory goes
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem_base, G::TMEM_COLS);
    }
}


// ------------------------------------------------------------------ two-CTA kernel
//
// Same stage, computed by CTA pairs (clusters of 2) with cta_group::2 MMAs on
// 256 x 256 tiles: each CTA stages 128 weight rows and 128 activation columns
// per k-block (32 KB instead of 48 KB for the same 4.2 MFLOP per CTA), which
// is what bounds the single-CTA version (L2 -> shared memory traffic). The
// pair's first CTA ("leader") owns the pipeline: its full barriers count the
// bytes both CTAs load, it alone issues the MMAs, and its commits arrive on
// the barriers of both CTAs. Each CTA's epilogue drains its own 128 TMEM
// lanes (output rows) and arrives on the leader's accumulator-empty barrier.

template <int OP>
__global__ void __launch_bounds__(kThreads, 1)
    tc_pair_kernel(const __grid_constant__ CUtensorMap tm_w, const __grid_constant__ CUtensorMap tm_x,
                   const __grid_constant__ CUtensorMap tm_wt,
                   const __grid_constant__ CUtensorMap tm_out, const StageArgs p)
{
    using T = OpTraits<OP>;
    using G = PairGeo<OP>;
    constexpr int S = G::STAGES;
    constexpr int BN = G::BN;

    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    Bars *bars = reinterpret_cast<Bars *>(smem + S * G::STAGE_BYTES + G::STAGING_BYTES);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t rank = cluster_ctarank();
    const bool leader = (rank == 0);
    const int pair = blockIdx.x >> 1;
    const int npairs = gridDim.x >> 1;
    const int tiles_m = (p.M + G::BM - 1) / G::BM;
    const int tiles_n = (p.N + BN - 1) / BN;
    const int num_tiles = tiles_m * tiles_n;
    const int num_kb = (p.K + G::BK - 1) / G::BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&bars->full[s], 1);
            mbar_init(&bars->empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&bars->acc_full[a], 1);
            mbar_init(&bars->acc_empty[a], 2 * 4);  // one arrival per epilogue warp, both CTAs
        }
        mbar_init(&bars->mma_done, 1);
        bars->abort = 0;
        fence_mbar_init();
    }
    if (warp == 0 && lane == 0) {
        tma_prefetch_desc(&tm_w);
        tma_prefetch_desc(&tm_x);
    }
    if (warp == 1) tmem_alloc_pair(&bars->tmem_base, G::TMEM_COLS);
    tc_fence_before();
    cluster_sync();  // both CTAs' barriers initialised and TMEM allocated
    tc_fence_after();
    const uint32_t tmem_base = bars->tmem_base;

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer (both CTAs)
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            uint32_t pending = 0, pending_ph = 0;  // leader: stages with loads in flight
            for (int t = pair; t < num_tiles; t += npairs) {
                const int m0p = (t / tiles_n) * G::BM;
                const int n0 = (t % tiles_n) * BN;
                // boxes past the matrix edge are not loaded (they only feed rows or
                // columns that are never stored); both CTAs count them the same way
                int tx = 0, my_boxes = 0;
                bool my_a = false;
                for (int r = 0; r < 2; ++r) {
                    const bool a_in = m0p + 128 * r < p.M;
                    int nb = 0;
                    for (int j = 0; j < G::NBOX; ++j)
                        if (n0 + (BN / 2) * r + j * G::BOX_N < p.N) ++nb;
                    tx += (a_in ? G::A_BYTES : 0) + nb * G::BOX_BYTES;
                    if (r == (int)rank) {
                        my_a = a_in;
                        my_boxes = nb;
                    }
                }
                for (int kb = 0; kb < num_kb; ++kb) {
                    if (!mbar_wait(&bars->empty[s], ph ^ 1, p.status, KERR_WAIT_EMPTY)) {
                        set_abort(bars);
                        goto producer_done;
                    }
                    uint8_t *st = smem + s * G::STAGE_BYTES;
                    const uint32_t full_leader = mapa_shared(smem_u32(&bars->full[s]), 0);
                    if (leader) mbar_arrive_expect_tx(&bars->full[s], (uint32_t)tx);
                    const int k0 = kb * G::BK;
                    if (my_a) {
                        const int ma = m0p + 128 * (int)rank;
                        if (tile_has_tail(p, ma))
                            tma_load_2d_pair(st, &tm_wt, full_leader, k0, ma - p.tail_row0);
                        else
                            tma_load_2d_pair(st, &tm_w, full_leader, k0, ma);
                    }
                    for (int j = 0; j < my_boxes; ++j)
                        tma_load_2d_pair(st + G::A_BYTES + j * G::BOX_BYTES, &tm_x, full_leader,
                                         n0 + (BN / 2) * (int)rank + j * G::BOX_N, k0);
                    if (leader) {
                        pending |= 1u << s;
                        pending_ph = (pending_ph & ~(1u << s)) | (ph << s);
                    }
                    if (++s == S) {
                        s = 0;
                        ph ^= 1;
                    }
                }
                if (aborted(bars)) break;
            }
        producer_done:
            // the leader's full barriers also count the peer's bytes: once they
            // complete, no copy of either CTA is still in flight
            for (int st = 0; st < S; ++st)
                if (pending & (1u << st))
                    mbar_wait(&bars->full[st], (pending_ph >> st) & 1u, p.status, KERR_WAIT_FULL);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer (leader only)
        if (lane == 0 && leader) {
            int s = 0;
            uint32_t ph = 0;
            int acc = 0;
            uint32_t acc_ph = 0;
            for (int t = pair; t < num_tiles; t += npairs) {
                if (!mbar_wait(&bars->acc_empty[acc], acc_ph ^ 1, p.status, KERR_WAIT_ACC_EMPTY)) {
                    set_abort(bars);
                    break;
                }
                tc_fence_after();
                const uint32_t d_tmem = tmem_base + acc * BN;
                bool ok = true;
                for (int kb = 0; kb < num_kb; ++kb) {
                    if (!mbar_wait(&bars->full[s], ph, p.status, KERR_WAIT_FULL)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a_addr = smem_u32(smem + s * G::STAGE_BYTES);
                    const uint32_t b_addr = a_addr + G::A_BYTES;
#pragma unroll
                    for (int k = 0; k < G::MMAS_PER_STAGE; ++k) {
                        const uint64_t ad =
                            smem_desc(a_addr + k * G::MMA_K_BYTES, 16, 1024, SMEM_SW128);
                        const uint64_t bd = smem_desc(b_addr + k * G::B_KSTEP_BYTES, G::BOX_BYTES,
                                                      1024, SMEM_SW128);
                        tc_mma_pair<T::kind>(d_tmem, ad, bd, G::idesc, (kb | k) != 0);
                    }
                    tc_commit_pair(&bars->empty[s], 0x3);  // stage free in both CTAs
                    if (++s == S) {
                        s = 0;
                        ph ^= 1;
                    }
                }
                if (!ok) {
                    set_abort(bars);
                    break;
                }
                tc_commit_pair(&bars->acc_full[acc], 0x3);  // accumulator ready in both CTAs
                if (++acc == 2) {
                    acc = 0;
                    acc_ph ^= 1;
                }
                if (aborted(bars)) break;
            }
            tc_commit_pair(&bars->mma_done, 0x1);
            mbar_wait(&bars->mma_done, 0, p.status, KERR_WAIT_FULL);
        }
    } else {
        // ------------------------------------------------------------ epilogue (warps 2..5, both CTAs)
        const int quarter = warp & 3;
        int acc = 0;
        uint32_t acc_ph = 0;
        uint8_t *staging = smem + S * G::STAGE_BYTES + (warp - 2) * 2 * kStageBufBytes;
        int sbuf = 0;
        for (int t = pair; t < num_tiles; t += npairs) {
            if (!mbar_wait(&bars->acc_full[acc], acc_ph, p.status, KERR_WAIT_ACC_FULL)) {
                set_abort(bars);
                break;
            }
            tc_fence_after();
            const int m0 = (t / tiles_n) * G::BM + 128 * (int)rank;
            const int n0 = (t % tiles_n) * BN;
            const uint32_t t_row = tmem_base + acc * BN + ((uint32_t)(quarter * 32) << 16);
            drain_warp<OP, BN>(p, &tm_out, t_row, lane, m0 + quarter * 32, n0, staging, sbuf);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive_cluster(mapa_shared(smem_u32(&bars->acc_empty[acc]), 0));
            if (++acc == 2) {
                acc = 0;
                acc_ph ^= 1;
            }
            if (aborted(bars)) break;
        }
    }

    if (warp >= 2 && lane == 0) bulk_wait<0>();  // staged stores done before shared memory goes
    tc_fence_before();
    __syncthreads();
    cluster_sync();  // both CTAs done with TMEM and shared memory
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc_pair(tmem_base, G::TMEM_COLS);
    }
}

// ------------------------------------------------------------------ launchers

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
    if (OP == OP_I8 && a.tail_hi > a.tail_lo) {
        if (!make_map(&twl, dt, T::elt, a.w_tail, a.M - a.tail_row0, a.K, a.ld_w_tail, G::BK, kBM))
            return cudaErrorInvalidValue;
        txl = tx;
    } else if (T::split) {
        if (!make_map(&twl, dt, T::elt, a.w_lo, a.M, a.K, a.ld_w, G::BK, kBM)) return cudaErrorInvalidValue;
        if (!make_map(&txl, dt, T::elt, a.x_lo, a.K, a.N, a.ld_x, G::BOX_N, G::BK, bswz))
            return cudaErrorInvalidValue;
    } else {
        twl = tw;
        txl = tx;
    }
    // bit per device: the attribute is per context. Set under a lock, since
    // callers on several host threads (the allocation-free entry point takes no
    // library lock) may reach here at once.
    static std::mutex attr_mu;
    static unsigned long long attr_set = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> lk(attr_mu);
        if (!(attr_set & (1ull << (dev & 63)))) {
            cudaError_t e = cudaFuncSetAttribute(
                tc_stage_kernel<OP>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM_BYTES);
            if (e != cudaSuccess) return e;
            attr_set |= 1ull << (dev & 63);
        }
    }
    const int tiles = ((a.M + kBM - 1) / kBM) * ((a.N + T::BN - 1) / T::BN);
    const int grid = tiles < num_sms ? tiles : num_sms;
    StageArgs b = a;
    CUtensorMap to;
    CUtensorMap to2;
    if (b.epi == EPI_TF32SPLIT) {
        // the next stage's (hi, lo) inputs: FP32 rows of 16-byte multiples
        const bool ok = ((uintptr_t)b.out & 15) == 0 && ((uintptr_t)b.out_lo & 15) == 0 &&
                        (b.ld_out * 4) % 16 == 0 &&
                        make_map(&to, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, b.out, b.M, b.N,
                                 b.ld_out, 32, 32) &&
                        make_map(&to2, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, b.out_lo, b.M, b.N,
                                 b.ld_out, 32, 32);
        b.tma_store = ok ? 1 : 0;
    } else {
        b.tma_store = make_out_map(&to, b) ? 1 : 0;
    }
    if (!b.tma_store) to = tw;
    if (b.epi != EPI_TF32SPLIT || !b.tma_store) to2 = to;
    tc_stage_kernel<OP><<<grid, kThreads, G::SMEM_BYTES, s>>>(tw, tx, twl, txl, to, to2, b);
    return cudaGetLastError();
}

template <int OP>
static cudaError_t launch_pair(const StageArgs &a, int num_sms, cudaStream_t s)
{
    using T = OpTraits<OP>;
    using G = PairGeo<OP>;
    CUtensorMapDataType dt = OP == OP_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                           : CU_TENSOR_MAP_DATA_TYPE_UINT8;
    CUtensorMap tw, tx, twt;
    if (!make_map(&tw, dt, T::elt, a.w, a.M, a.K, a.ld_w, G::BK, 128)) return cudaErrorInvalidValue;
    if (!make_map(&tx, dt, T::elt, a.x, a.K, a.N, a.ld_x, G::BOX_N, G::BK)) return cudaErrorInvalidValue;
    if (a.tail_hi > a.tail_lo) {
        if (!make_map(&twt, dt, T::elt, a.w_tail, a.M - a.tail_row0, a.K, a.ld_w_tail, G::BK, 128))
            return cudaErrorInvalidValue;
    } else {
        twt = tw;
    }
    // Per device, once, under a lock (see launch_op): the shared-memory attribute
    // and the occupancy-derived pair count, published together.
    static std::mutex attr_mu;
    static unsigned long long attr_set = 0;
    static int max_pairs[64];
    int dev = 0;
    cudaGetDevice(&dev);
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = G::SMEM_BYTES;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int cap = 0;
    {
        std::lock_guard<std::mutex> lk(attr_mu);
        if (!(attr_set & (1ull << (dev & 63)))) {
            cudaError_t e = cudaFuncSetAttribute(
                tc_pair_kernel<OP>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM_BYTES);
            if (e != cudaSuccess) return e;
            int clusters = 0;
            cfg.gridDim = dim3(2 * (num_sms / 2));
            e = cudaOccupancyMaxActiveClusters(&clusters, tc_pair_kernel<OP>, &cfg);
            if (e != cudaSuccess || clusters < 1) {
                cudaGetLastError();
                clusters = num_sms / 2;
            }
            max_pairs[dev & 63] = clusters;
            attr_set |= 1ull << (dev & 63);
        }
        cap = max_pairs[dev & 63];
    }
    const int tiles = ((a.M + G::BM - 1) / G::BM) * ((a.N + G::BN - 1) / G::BN);
    const int pairs = tiles < cap ? tiles : cap;
    cfg.gridDim = dim3(2 * pairs);
    StageArgs b = a;
    CUtensorMap to;
    b.tma_store = make_out_map(&to, b) ? 1 : 0;
    if (!b.tma_store) to = tw;
    return cudaLaunchKernelEx(&cfg, tc_pair_kernel<OP>, tw, tx, twt, to, b);
}

// Two-CTA tiles for BF16 and INT8 unless FG_CTA_PAIR=0.
static bool use_pairs()
{
    static const bool on = [] {
        const char *v = getenv("FG_CTA_PAIR");
        return !(v && v[0] == '0');
    }();
    return on;
}

cudaError_t launch_tc_stage(const StageArgs &a, int num_sms, cudaStream_t s)
{
    if (a.M <= 0 || a.N <= 0 || a.K <= 0) return cudaErrorInvalidValue;
    switch (a.op) {
    case OP_BF16: return use_pairs() ? launch_pair<OP_BF16>(a, num_sms, s) : launch_op<OP_BF16>(a, num_sms, s);
    case OP_I8: return use_pairs() ? launch_pair<OP_I8>(a, num_sms, s) : launch_op<OP_I8>(a, num_sms, s);
    case OP_TF32X3: return launch_op<OP_TF32X3>(a, num_sms, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace fg
