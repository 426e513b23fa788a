// Grouped GEMM stages on single CTAs (sm_100a): the stages of many chains in
// one persistent launch, each CTA working through its own list of tiles, a tile
// waiting only for the column block of the stage it reads.
//
// This is the kernel behind grouped launches of 3xTF32 (FP32) chains and the
// single-CTA option for BF16 / INT8 groups, whose small stages (dimensions from
// 64) waste most of a 256 x 256 pair tile. Per CTA, 6 warps as in the one-stage
// kernel (fg_gemm_tc.cu): warp 0 TMA producer, warp 1 TMEM owner and MMA issuer,
// warps 2-5 epilogue, two TMEM accumulators. Per tile the producer first
// acquires the column-block counter of the stage it reads (released by that
// stage's epilogue warps once their stores are in memory), so that a chain's
// next stage starts on a column block as soon as that block is complete,
// while other chains' tiles keep the remaining CTAs busy.
//
// Tables (stage descriptors with their tensor maps, per-CTA work lists) live
// in device memory, built once per group shape on the host; every wait is
// bounded (fg_ptx.cuh) and reports its cause in the status word.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <queue>
#include <vector>

#include "fg_tc_common.cuh"

namespace fg {

// Tile geometry of a single-CTA grouped kernel: 128 weight rows x BN
// activation columns, an S-deep ring of TMA stages.
template <int OP, int BN_, int S_>
struct GroupGeo {
    using T = OpTraits<OP>;
    static constexpr int BN = BN_;
    static constexpr int S = S_;
    static constexpr int BK = kRowBytes / T::elt;
    static constexpr int A_BYTES = kBM * kRowBytes;
    static constexpr int BOX_N = kRowBytes / T::elt;
    static constexpr int BOX_BYTES = BOX_N * BK * T::elt;
    static constexpr int NBOX = BN / BOX_N;
    static constexpr int B_BYTES = NBOX * BOX_BYTES;
    static constexpr int PARTS = T::split ? 2 : 1;
    static constexpr int STAGE_BYTES = PARTS * (A_BYTES + B_BYTES);
    static constexpr int MMA_K_BYTES = 32;
    static constexpr int MMAS_PER_STAGE = kRowBytes / MMA_K_BYTES;
    static constexpr int B_KSTEP_BYTES = (MMA_K_BYTES / T::elt) * kRowBytes;
    static constexpr int B_SBO = T::b_layout == SMEM_SW128_32B ? 512 : 1024;
    // TMEM: two accumulators of BN columns; 3xTF32 adds two correction
    // accumulators (hi*lo + lo*hi, one per tile in flight) at CORR_COLS
    static constexpr int ACC_COLS = BN;
    static constexpr int CORR_COLS = 2 * BN;
    static constexpr int TMEM_COLS = (T::split ? 4 : 2) * BN;
    static constexpr int STAGING_BYTES = kEpiStagingBytes;
    static constexpr int SMEM_BYTES = S * STAGE_BYTES + STAGING_BYTES + 1024 + 256;
    static constexpr uint32_t idesc = OP == OP_BF16 ? make_idesc(1, 1, 1, 0, 1, kBM, BN)
                                    : OP == OP_I8   ? make_idesc(2, 0, 1, 0, 1, kBM, BN)
                                                    : make_idesc(1, 2, 2, 0, 1, kBM, BN);
    static_assert(SMEM_BYTES <= 232448, "shared memory per CTA");
    static_assert(TMEM_COLS <= 512, "TMEM columns");
    static_assert(S <= (T::split ? 6 : 8), "barrier slots (3xTF32 uses the last two pairs)");
};

struct alignas(64) GroupStage {
    CUtensorMap tm_w;    // weights (3xTF32: hi), box 128 rows x 128 bytes
    CUtensorMap tm_x;    // activations (3xTF32: hi), MN-major boxes of 128 bytes
    CUtensorMap tm_w2;   // INT8: the pre-shifted tail block; 3xTF32: weights lo
    CUtensorMap tm_x2;   // 3xTF32: activations lo
    CUtensorMap tm_out;  // output, for the staged (TMA-store) epilogue
    CUtensorMap tm_out2; // 3xTF32 between stages: the lo half of the output
    StageArgs a;
    int tiles_m, tiles_n;
    int prev;            // stage whose output this one reads (-1: none)
    int done_off;        // this stage's column-block counters
};

struct GroupArgs {
    const GroupStage *st;
    const WorkEntry *sched;
    const int *off;  // static lists: CTA c runs sched[off[c] .. off[c + 1])
    int *done;
    int *status;
    int dynamic;     // 1: one list sched[0 .. total) in dependency order, taken in turn
    int total;       //    by the CTAs through the counter *next (zeroed with `done`)
    int *next;
};

// Entries a CTA's producer has taken, handed in order to its MMA warp and
// epilogue warps (dynamic lists). Lives in the bytes after Bars.
constexpr int kRing = 4;
struct EntryRing {
    uint64_t full[kRing];   // the producer published entry[slot]
    uint64_t empty[kRing];  // the MMA warp and the 4 epilogue warps have read it
    int entry[kRing];       // work entry index, -1: no more work
};
static_assert(sizeof(Bars) + sizeof(EntryRing) <= 256, "barrier block");

// Epilogue warps per CTA: counter increments per finished tile.
constexpr int kGroupDonePerTile = 4;

template <int OP, int BN, int S>
__global__ void __launch_bounds__(kThreads, 1) tc_group_kernel(const GroupArgs g)
{
    using T = OpTraits<OP>;
    using G = GroupGeo<OP, BN, S>;

    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    Bars *bars = reinterpret_cast<Bars *>(smem + S * G::STAGE_BYTES + G::STAGING_BYTES);

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    int *status = g.status;
    const int q_begin = g.dynamic ? 0 : g.off[blockIdx.x];
    const int q_end = g.dynamic ? 0 : g.off[blockIdx.x + 1];
    EntryRing *ring = reinterpret_cast<EntryRing *>(reinterpret_cast<uint8_t *>(bars) + sizeof(Bars));
    // k-th entry of this CTA (static list) or of its ring (dynamic): -1 when done,
    // -2 when a wait ran out
    auto take = [&](int k, bool release, int code) -> int {
        if (!g.dynamic) return q_begin + k < q_end ? q_begin + k : -1;
        const int slot = k % kRing;
        const uint32_t rph = (uint32_t)(k / kRing) & 1u;
        if (!mbar_wait(&ring->full[slot], rph, status, code)) return -2;
        const int q = *reinterpret_cast<volatile int *>(&ring->entry[slot]);
        if (release) mbar_arrive(&ring->empty[slot]);
        return q;
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&bars->full[s], 1);
            mbar_init(&bars->empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&bars->acc_full[a], 1);
            mbar_init(&bars->acc_empty[a], kGroupDonePerTile);  // one arrival per epilogue warp
        }
        if constexpr (T::split)
            for (int a = 0; a < 2; ++a) {
                mbar_init(&bars->full[6 + a], 1);                    // correction ready
                mbar_init(&bars->empty[6 + a], kGroupDonePerTile);   // correction drained
            }
        for (int i = 0; i < kRing; ++i) {
            mbar_init(&ring->full[i], 1);
            mbar_init(&ring->empty[i], 1 + kGroupDonePerTile);
        }
        mbar_init(&bars->mma_done, 1);
        bars->abort = 0;
        fence_mbar_init();
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
            uint32_t pending = 0, pending_ph = 0;
            int last_si = -1;
            for (int k = 0;; ++k) {
                int q;
                if (g.dynamic) {
                    // take the next entry of the global list and publish it to this
                    // CTA's MMA and epilogue warps
                    const int slot = k % kRing;
                    const uint32_t rph = (uint32_t)(k / kRing) & 1u;
                    if (!mbar_wait(&ring->empty[slot], rph ^ 1, status, KERR_WAIT_EMPTY)) {
                        set_abort(bars);
                        goto producer_done;
                    }
                    q = atomicAdd(g.next, 1);
                    if (q >= g.total) q = -1;
                    *reinterpret_cast<volatile int *>(&ring->entry[slot]) = q;
                    mbar_arrive(&ring->full[slot]);
                } else {
                    q = q_begin + k < q_end ? q_begin + k : -1;
                }
                if (q < 0) break;
                const WorkEntry e = g.sched[q];
                const int si = (int)e.stage;
                const int mb = (int)(e.mbnb >> 16), nb = (int)(e.mbnb & 0xffffu);
                const GroupStage &cs = g.st[si];
                const int N = cs.a.N;
                const int num_kb = (cs.a.K + G::BK - 1) / G::BK;
                const int prev = cs.prev;
                if (si != last_si) {
                    tma_prefetch_desc(&cs.tm_w);
                    tma_prefetch_desc(&cs.tm_x);
                    if (T::split || OP == OP_I8) tma_prefetch_desc(&cs.tm_w2);
                    if (T::split) tma_prefetch_desc(&cs.tm_x2);
                    last_si = si;
                }
                if (prev >= 0) {
                    // every tile of column block nb of the stage read here is stored
                    const GroupStage &ps = g.st[prev];
                    const int *cnt = g.done + ps.done_off + nb;
                    const int need = kGroupDonePerTile * ps.tiles_m;
                    if (ld_acquire_gpu(cnt) < need) {
                        const uint64_t t0 = globaltimer_ns();
                        while (ld_acquire_gpu(cnt) < need) {
                            __nanosleep(64);
                            if (wait_expired(t0)) {
                                atomicCAS(status, 0, KERR_WAIT_DEPENDENCY);
                                set_abort(bars);
                                goto producer_done;
                            }
                        }
                    }
                    fence_proxy_async_global();  // generic-proxy stores before the TMA reads
                }
                {
                    const int m0 = mb * kBM;
                    const int n0 = nb * BN;
                    // boxes that start past the last column are not loaded: they only
                    // feed output columns that are never stored
                    int nvb = (N - n0 + G::BOX_N - 1) / G::BOX_N;
                    nvb = nvb < G::NBOX ? nvb : G::NBOX;
                    const uint32_t tx = G::PARTS * (G::A_BYTES + nvb * G::BOX_BYTES);
                    const bool a_tail = OP == OP_I8 && tile_has_tail(cs.a, m0);
                    const CUtensorMap *tm_a = a_tail ? &cs.tm_w2 : &cs.tm_w;
                    const int a_row = a_tail ? m0 - cs.a.tail_row0 : m0;
                    const CUtensorMap *tm_b = &cs.tm_x;
                    const CUtensorMap *tm_a2 = &cs.tm_w2;
                    const CUtensorMap *tm_b2 = &cs.tm_x2;
                    for (int kb = 0; kb < num_kb; ++kb) {
                        if (!mbar_wait(&bars->empty[s], ph ^ 1, status, KERR_WAIT_EMPTY)) {
                            set_abort(bars);
                            goto producer_done;
                        }
                        uint8_t *st = smem + s * G::STAGE_BYTES;
                        mbar_arrive_expect_tx(&bars->full[s], tx);
                        const int k0 = kb * G::BK;
                        tma_load_2d(st, tm_a, &bars->full[s], k0, a_row);
                        for (int j = 0; j < nvb; ++j)
                            tma_load_2d(st + G::A_BYTES + j * G::BOX_BYTES, tm_b, &bars->full[s],
                                        n0 + j * G::BOX_N, k0);
                        if constexpr (T::split) {
                            uint8_t *st2 = st + G::A_BYTES + G::B_BYTES;
                            tma_load_2d(st2, tm_a2, &bars->full[s], k0, m0);
                            for (int j = 0; j < nvb; ++j)
                                tma_load_2d(st2 + G::A_BYTES + j * G::BOX_BYTES, tm_b2,
                                            &bars->full[s], n0 + j * G::BOX_N, k0);
                        }
                        pending |= 1u << s;
                        pending_ph = (pending_ph & ~(1u << s)) | (ph << s);
                        if (++s == S) {
                            s = 0;
                            ph ^= 1;
                        }
                    }
                }
                if (aborted(bars)) break;
            }
        producer_done:
            // never leave with copies in flight into this CTA's shared memory
            for (int st = 0; st < S; ++st)
                if (pending & (1u << st))
                    mbar_wait(&bars->full[st], (pending_ph >> st) & 1u, status, KERR_WAIT_FULL);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            int acc = 0;
            uint32_t acc_ph = 0;
            int cb = 0;          // 3xTF32: correction accumulator of this tile
            uint32_t cb_ph = 0;
            for (int k = 0;; ++k) {
                const int q = take(k, true, KERR_WAIT_FULL);
                if (q == -2) {
                    set_abort(bars);
                    goto mma_done;
                }
                if (q < 0) break;
                const GroupStage &cs = g.st[g.sched[q].stage];
                const int num_kb = (cs.a.K + G::BK - 1) / G::BK;
                // 3xTF32 hands the hi*hi partial sum to the epilogue every kchunk
                // k-blocks (FP32 promotion in registers, as in the one-stage kernel);
                // the small hi*lo + lo*hi terms accumulate over the whole tile
                const int kchunk = (T::split && cs.a.kchunk > 0) ? cs.a.kchunk : num_kb;
                uint32_t c_tmem = 0;
                if constexpr (T::split) {
                    if (!mbar_wait(&bars->empty[6 + cb], cb_ph ^ 1, status, KERR_WAIT_ACC_EMPTY)) {
                        set_abort(bars);
                        goto mma_done;
                    }
                    tc_fence_after();
                    c_tmem = tmem_base + G::CORR_COLS + cb * BN;
                }
                for (int kc = 0; kc < num_kb; kc += kchunk) {
                    if (!mbar_wait(&bars->acc_empty[acc], acc_ph ^ 1, status,
                                   KERR_WAIT_ACC_EMPTY)) {
                        set_abort(bars);
                        goto mma_done;
                    }
                    tc_fence_after();
                    const uint32_t d_tmem = tmem_base + acc * G::ACC_COLS;
                    const int kend = kc + kchunk < num_kb ? kc + kchunk : num_kb;
                    for (int kb = kc; kb < kend; ++kb) {
                        if (!mbar_wait(&bars->full[s], ph, status, KERR_WAIT_FULL)) {
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
                                tc_mma<T::kind>(c_tmem, ad, bd_lo, G::idesc, (kb | k) != 0);
                                tc_mma<T::kind>(c_tmem, ad_lo, bd, G::idesc, 1);
                                tc_mma<T::kind>(d_tmem, ad, bd, G::idesc, accumulate);
                            } else {
                                tc_mma<T::kind>(d_tmem, ad, bd, G::idesc, accumulate);
                            }
                        }
                        tc_commit(&bars->empty[s]);
                        if (++s == S) {
                            s = 0;
                            ph ^= 1;
                        }
                    }
                    tc_commit(&bars->acc_full[acc]);
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
            tc_commit(&bars->mma_done);
            mbar_wait(&bars->mma_done, 0, status, KERR_WAIT_FULL);
        }
    } else {
        // ------------------------------------------------------------ epilogue (warps 2..5)
        const int quarter = warp & 3;
        int acc = 0;
        uint32_t acc_ph = 0;
        int cb = 0;
        uint32_t cb_ph = 0;
        uint8_t *staging = smem + S * G::STAGE_BYTES + (warp - 2) * 2 * kStageBufBytes;
        int sbuf = 0;
        for (int k = 0;; ++k) {
            const int q = take(k, false, KERR_WAIT_ACC_FULL);
            if (g.dynamic) {
                __syncwarp();
                if (lane == 0 && q != -2) mbar_arrive(&ring->empty[k % kRing]);
            }
            if (q == -2) {
                set_abort(bars);
                break;
            }
            if (q < 0) break;
            const WorkEntry e = g.sched[q];
            const int mb = (int)(e.mbnb >> 16), nb = (int)(e.mbnb & 0xffffu);
            const GroupStage &cs = g.st[e.stage];
            const int m0 = mb * kBM;
            const int n0 = nb * BN;
            bool ok = true;
            if constexpr (T::split) {
                const int num_kb = (cs.a.K + G::BK - 1) / G::BK;
                const int kchunk = cs.a.kchunk > 0 ? cs.a.kchunk : num_kb;
                const int row = m0 + quarter * 32 + lane;
                float sum[BN / 32][32];
#pragma unroll
                for (int c = 0; c < BN / 32; ++c)
#pragma unroll
                    for (int j = 0; j < 32; ++j) sum[c][j] = 0.f;
                for (int kc = 0; kc < num_kb; kc += kchunk) {
                    if (!mbar_wait(&bars->acc_full[acc], acc_ph, status, KERR_WAIT_ACC_FULL)) {
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
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&bars->acc_empty[acc]);
                    if (++acc == 2) {
                        acc = 0;
                        acc_ph ^= 1;
                    }
                }
                // the tile's correction terms, added once
                if (ok && !mbar_wait(&bars->full[6 + cb], cb_ph, status, KERR_WAIT_ACC_FULL))
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
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&bars->empty[6 + cb]);
                    if (++cb == 2) {
                        cb = 0;
                        cb_ph ^= 1;
                    }
                }
                if (ok && cs.a.tma_store) {
                    // staged TMA stores, 32 columns at a time: the FP32 result, or the
                    // (hi, lo) TF32 pair of the next stage's input in the two buffers
                    const int warp_row0 = m0 + quarter * 32;
                    const bool rows_in = warp_row0 < cs.a.M;
                    const bool split_out = cs.a.epi == EPI_TF32SPLIT;
#pragma unroll
                    for (int c = 0; c < BN / 32; ++c) {
                        const int nc = n0 + c * 32;
                        if (nc >= cs.a.N) break;  // warp-uniform
                        uint8_t *b0 = staging + (split_out ? 0 : sbuf) * kStageBufBytes;
                        uint8_t *b1 = staging + kStageBufBytes;
                        if (lane == 0) {
                            if (split_out)
                                bulk_wait_read<0>();  // both buffers' last stores have read them
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
                            tma_store_2d(&cs.tm_out, b0, nc, warp_row0);
                            if (split_out) tma_store_2d(&cs.tm_out2, b1, nc, warp_row0);
                            bulk_commit();
                        }
                    }
                } else if (ok) {
#pragma unroll
                    for (int c = 0; c < BN / 32; ++c) {
                        const int nc = n0 + c * 32;
                        if (nc < cs.a.N && row < cs.a.M) {
                            uint32_t v[32];
#pragma unroll
                            for (int j = 0; j < 32; ++j) v[j] = __float_as_uint(sum[c][j]);
                            store_chunk<OP>(cs.a, row, nc, v);
                        }
                    }
                }
            } else {
                if (!mbar_wait(&bars->acc_full[acc], acc_ph, status, KERR_WAIT_ACC_FULL)) {
                    ok = false;
                } else {
                    tc_fence_after();
                    const uint32_t t_row =
                        tmem_base + acc * G::ACC_COLS + ((uint32_t)(quarter * 32) << 16);
                    drain_warp<OP, BN>(cs.a, &cs.tm_out, t_row, lane, m0 + quarter * 32, n0,
                                       staging, sbuf);
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&bars->acc_empty[acc]);
                    if (++acc == 2) {
                        acc = 0;
                        acc_ph ^= 1;
                    }
                }
            }
            if (!ok) {
                set_abort(bars);
                break;
            }
            // direct stores of this lane before the release (TMA stores are ordered
            // by lane 0's bulk wait and fences below)
            if (!cs.a.tma_store) __threadfence();
            __syncwarp();
            if (lane == 0) {
                // this warp's rows of the tile are in memory: release them
                bulk_wait<0>();
                fence_proxy_async_global();
                __threadfence();
                red_release_gpu_add(g.done + cs.done_off + nb, 1);
            }
            if (aborted(bars)) break;
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

// ------------------------------------------------------------------ scheduling (host)

void list_schedule(const SchedStage *st, int n, int units, double handoff, std::vector<int> &off,
                   std::vector<WorkEntry> &entries, double *makespan, std::vector<double> *starts,
                   const SchedOpts *opts)
{
    SchedOpts o;
    if (opts) o = *opts;
    const bool feeding = o.feed_stage >= 0 && o.feed_stage < n && o.feed_workers > 0 &&
                         o.feed_workers < units && o.feed_rows > 0;
    double span = 0.0;
    std::vector<int> depth(n, 0), order(n);
    long total = 0, nblocks = 0;
    int max_tn = 0;
    for (int i = 0; i < n; ++i) {
        depth[i] = st[i].prev < 0 ? 0 : depth[st[i].prev] + 1;
        order[i] = i;
        total += (long)st[i].tiles_m * st[i].tiles_n;
        max_tn = std::max(max_tn, st[i].tiles_n);
        nblocks = std::max<long>(nblocks, (long)st[i].done_off +
                                              (long)st[i].tiles_n * (st[i].row_done ? st[i].tiles_m : 1));
    }
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return depth[x] < depth[y]; });

    // ---- the placement order: windows of column blocks, stages in depth order,
    // each stage's tiles column block by column block (or row tile by row tile);
    // a fed stage's deferred rows after its other tiles
    struct Item {
        int si, mb, nb;
        int u_lo, u_hi;  // workers that may take it
    };
    std::vector<Item> items;
    items.reserve(total);
    const int W = o.window > 0 ? o.window : (max_tn > 0 ? max_tn : 1);
    for (int w0 = 0; w0 < std::max(max_tn, 1); w0 += W)
        for (int si : order) {
            const SchedStage &c = st[si];
            const int n0 = std::min(w0, c.tiles_n), n1 = std::min(w0 + W, c.tiles_n);
            const int nw = n1 - n0;
            if (nw <= 0) continue;
            const bool fed = feeding && si == o.feed_stage;
            const bool reads_fed = feeding && c.prev == o.feed_stage;
            const int defer = fed ? std::min(o.feed_rows, c.tiles_m) : 0;
            const int kept = c.tiles_m - defer;
            const int hi = reads_fed || fed ? units - o.feed_workers : units;
            for (long it = 0; it < (long)kept * nw; ++it) {
                const int nb = n0 + (int)(c.row_major ? it % nw : it / kept);
                const int mb = (int)(c.row_major ? it / nw : it % kept);
                items.push_back(Item{si, mb, nb, 0, hi});
            }
            for (long it = 0; it < (long)defer * nw; ++it)  // feeders only
                items.push_back(Item{si, kept + (int)(it / nw), n0 + (int)(it % nw),
                                     units - o.feed_workers, units});
        }

    // ---- placement: each tile to the allowed worker that can start it first
    std::vector<double> block_done(nblocks, 0.0);
    std::vector<std::vector<WorkEntry>> per(units);
    std::vector<std::vector<double>> per_start(starts ? units : 0);
    // Small problems (one chain's few hundred tiles) or restricted workers: scan
    // the allowed workers, ties to the lowest index. Larger ones: a heap of (free
    // time, worker), O(log workers) per tile; a tile whose input is not ready
    // before the earliest free worker takes that worker.
    const bool scan = feeding || (double)units * (double)total <= 2e5;
    std::vector<double> free_at(units, 0.0);
    using Slot = std::pair<double, int>;
    std::priority_queue<Slot, std::vector<Slot>, std::greater<Slot>> heap;
    if (!scan)
        for (int u = 0; u < units; ++u) heap.push({0.0, u});
    for (const Item &t : items) {
        const SchedStage &c = st[t.si];
        const int nb = t.nb, mb = t.mb;
        double ready = 0.0;
        if (c.prev >= 0) {
            const SchedStage &p = st[c.prev];
            if (!p.row_done) {
                ready = block_done[p.done_off + nb] + handoff;
            } else {
                const double *rd = &block_done[p.done_off + (long)nb * p.tiles_m];
                for (int g = 0; g < p.tiles_m; ++g)
                    ready = std::max(ready, rd[g] + handoff - (c.stream > 0 ? g * c.stream : 0.0));
            }
        }
        int best = t.u_lo;
        double start;
        if (scan) {
            start = 1e300;
            for (int u = t.u_lo; u < t.u_hi; ++u) {
                const double tu = free_at[u] > ready ? free_at[u] : ready;
                if (tu < start - 1e-9) start = tu, best = u;
            }
        } else {
            const Slot top = heap.top();
            heap.pop();
            best = top.second;
            start = top.first > ready ? top.first : ready;
        }
        const double fin = start + c.cost;
        if (scan)
            free_at[best] = fin;
        else
            heap.push({fin, best});
        per[best].push_back(WorkEntry{(uint32_t)t.si, ((uint32_t)mb << 16) | (uint32_t)nb});
        if (starts) per_start[best].push_back(start);
        double &bd = block_done[c.done_off + (c.row_done ? (long)nb * c.tiles_m + mb : nb)];
        if (fin > bd) bd = fin;
        if (fin > span) span = fin;
    }
    if (makespan) *makespan = span;
    off.assign(units + 1, 0);
    entries.clear();
    entries.reserve(total);
    if (starts) starts->clear();
    for (int u = 0; u < units; ++u) {
        off[u + 1] = off[u] + (int)per[u].size();
        entries.insert(entries.end(), per[u].begin(), per[u].end());
        if (starts) starts->insert(starts->end(), per_start[u].begin(), per_start[u].end());
    }
}

// ------------------------------------------------------------------ planning and launch (host)

namespace {

// Dynamic lists for the single-CTA kernel (FG_GROUP_DYNAMIC=0: static per-CTA lists).
bool group_dynamic()
{
    static const bool on = [] {
        const char *v = getenv("FG_GROUP_DYNAMIC");
        return !(v && v[0] == '0');
    }();
    return on;
}

template <int OP, int BN, int S>
cudaError_t single_capacity(int num_sms, int &ctas)
{
    using G = GroupGeo<OP, BN, S>;
    static std::mutex mu;
    static int cap[64];
    static unsigned long long known = 0;
    std::lock_guard<std::mutex> lk(mu);
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(known & (1ull << (dev & 63)))) {
        cudaError_t e = cudaFuncSetAttribute(tc_group_kernel<OP, BN, S>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tc_group_kernel<OP, BN, S>,
                                                          kThreads, G::SMEM_BYTES);
        if (e != cudaSuccess || per_sm < 1) {
            cudaGetLastError();
            return cudaErrorNotSupported;
        }
        cap[dev & 63] = per_sm;
        known |= 1ull << (dev & 63);
    }
    ctas = cap[dev & 63] * num_sms;  // num_sms may be fewer than the device's: a cap
    return cudaSuccess;
}

template <int OP, int BN, int S>
cudaError_t plan_single(const StageArgs *stages, const int *prev, int n, int kernel, int num_sms,
                        GroupLaunch &out)
{
    using T = OpTraits<OP>;
    using G = GroupGeo<OP, BN, S>;
    const CUtensorMapDataType dt = OP == OP_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                 : OP == OP_I8   ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                                 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    const CUtensorMapSwizzle bswz = T::b_layout == SMEM_SW128_32B
                                        ? CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B
                                        : CU_TENSOR_MAP_SWIZZLE_128B;
    std::vector<GroupStage> st(n);
    std::vector<SchedStage> ss(n);
    long items = 0;
    int done_off = 0;
    for (int i = 0; i < n; ++i) {
        const StageArgs &a = stages[i];
        if (prev[i] >= i) return cudaErrorInvalidValue;
        GroupStage &cs = st[i];
        memset(&cs, 0, sizeof cs);
        if (!make_map(&cs.tm_w, dt, T::elt, a.w, a.M, a.K, a.ld_w, G::BK, kBM))
            return cudaErrorInvalidValue;
        if (!make_map(&cs.tm_x, dt, T::elt, a.x, a.K, a.N, a.ld_x, G::BOX_N, G::BK, bswz))
            return cudaErrorInvalidValue;
        cs.tm_w2 = cs.tm_w;
        cs.tm_x2 = cs.tm_x;
        if (OP == OP_I8 && a.tail_hi > a.tail_lo) {
            if (!make_map(&cs.tm_w2, dt, T::elt, a.w_tail, a.M - a.tail_row0, a.K, a.ld_w_tail,
                          G::BK, kBM))
                return cudaErrorInvalidValue;
        } else if (T::split) {
            if (!make_map(&cs.tm_w2, dt, T::elt, a.w_lo, a.M, a.K, a.ld_w, G::BK, kBM))
                return cudaErrorInvalidValue;
            if (!make_map(&cs.tm_x2, dt, T::elt, a.x_lo, a.K, a.N, a.ld_x, G::BOX_N, G::BK, bswz))
                return cudaErrorInvalidValue;
        }
        cs.a = a;
        if (a.epi == EPI_TF32SPLIT) {
            // the next stage's (hi, lo) inputs: FP32 rows of 16-byte multiples
            const bool ok = ((uintptr_t)a.out & 15) == 0 && ((uintptr_t)a.out_lo & 15) == 0 &&
                            (a.ld_out * 4) % 16 == 0 &&
                            make_map(&cs.tm_out, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.out, a.M,
                                     a.N, a.ld_out, 32, 32) &&
                            make_map(&cs.tm_out2, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.out_lo,
                                     a.M, a.N, a.ld_out, 32, 32);
            cs.a.tma_store = ok ? 1 : 0;
        } else {
            cs.a.tma_store = make_out_map(&cs.tm_out, cs.a) ? 1 : 0;
        }
        if (!cs.a.tma_store) cs.tm_out = cs.tm_out2 = cs.tm_w;
        cs.tiles_m = (a.M + kBM - 1) / kBM;
        cs.tiles_n = (a.N + BN - 1) / BN;
        if (cs.tiles_m > 65535 || cs.tiles_n > 65535) return cudaErrorNotSupported;
        cs.prev = prev[i];
        cs.done_off = done_off;
        done_off += cs.tiles_n;
        items += (long)cs.tiles_m * cs.tiles_n;
        const double kb = (double)((a.K + G::BK - 1) / G::BK);
        ss[i] = SchedStage{cs.tiles_m, cs.tiles_n, cs.prev, cs.done_off,
                           kb * (T::split ? 3.0 : 1.0) * (BN / 128.0) + 4.0};
    }
    int ctas = 0;
    cudaError_t e = single_capacity<OP, BN, S>(num_sms, ctas);
    if (e != cudaSuccess) return e;
    if (items < ctas) ctas = (int)items;
    std::vector<int> off;
    std::vector<WorkEntry> ent;
    std::vector<double> starts;
    const bool dyn = group_dynamic();
    list_schedule(ss.data(), n, ctas, 2.0, off, ent, nullptr, dyn ? &starts : nullptr);
    if (dyn) {
        // one list in order of the schedule's start times (every dependency
        // starts earlier, so it comes first), taken by the CTAs in turn
        std::vector<int> order(ent.size());
        for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
        std::stable_sort(order.begin(), order.end(),
                         [&](int x, int y) { return starts[x] < starts[y]; });
        std::vector<WorkEntry> sorted(ent.size());
        for (size_t i = 0; i < order.size(); ++i) sorted[i] = ent[order[i]];
        ent.swap(sorted);
        off.assign(ctas + 1, (int)items);
        off[0] = 0;
    }
    auto r = [](size_t b) { return (b + 255) & ~(size_t)255; };
    out.kernel = kernel;
    out.op = OP;
    out.ctas = ctas;
    out.entries = items;
    out.dynamic = dyn ? 1 : 0;
    out.done_ints = (size_t)done_off + 1;  // the last one: the dynamic list's counter
    out.off_st = 0;
    out.off_sched = r((size_t)n * sizeof(GroupStage));
    out.off_off = out.off_sched + r((size_t)items * sizeof(WorkEntry));
    out.tables.assign(out.off_off + r((size_t)(ctas + 1) * sizeof(int)), 0);
    memcpy(out.tables.data(), st.data(), (size_t)n * sizeof(GroupStage));
    memcpy(out.tables.data() + out.off_sched, ent.data(), (size_t)items * sizeof(WorkEntry));
    memcpy(out.tables.data() + out.off_off, off.data(), (size_t)(ctas + 1) * sizeof(int));
    return cudaSuccess;
}

template <int OP, int BN, int S>
cudaError_t launch_single(const GroupLaunch &g, const void *tables_dev, int *done, int *status,
                          cudaStream_t s)
{
    using G = GroupGeo<OP, BN, S>;
    const unsigned char *base = static_cast<const unsigned char *>(tables_dev);
    GroupArgs a;
    a.st = reinterpret_cast<const GroupStage *>(base + g.off_st);
    a.sched = reinterpret_cast<const WorkEntry *>(base + g.off_sched);
    a.off = reinterpret_cast<const int *>(base + g.off_off);
    a.done = done;
    a.status = status;
    a.dynamic = g.dynamic;
    a.total = (int)g.entries;
    a.next = done + g.done_ints - 1;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;  // all CTAs resident: they wait on one another
    attr[0].val.cooperative = 1;
    cfg.gridDim = dim3(g.ctas);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = G::SMEM_BYTES;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, tc_group_kernel<OP, BN, S>, a);
}

}  // namespace

int group_tile_n(int kernel, int op)
{
    if (op == OP_TF32X3) return 128;
    return kernel == GK_SINGLE_128 ? 128 : 256;
}

cudaError_t plan_single_group(const StageArgs *stages, const int *prev, int n, int kernel,
                              int num_sms, GroupLaunch &out)
{
    if (n < 1) return cudaErrorInvalidValue;
    for (int i = 0; i < n; ++i)
        if (stages[i].op != stages[0].op || stages[i].M <= 0 || stages[i].K <= 0 ||
            stages[i].N <= 0)
            return cudaErrorInvalidValue;
    const int op = stages[0].op;
    if (op == OP_TF32X3) return plan_single<OP_TF32X3, 128, 3>(stages, prev, n, GK_SINGLE_128, num_sms, out);
    if (kernel == GK_SINGLE_256) {
        if (op == OP_BF16) return plan_single<OP_BF16, 256, 4>(stages, prev, n, kernel, num_sms, out);
        if (op == OP_I8) return plan_single<OP_I8, 256, 4>(stages, prev, n, kernel, num_sms, out);
    } else if (kernel == GK_SINGLE_128) {
        if (op == OP_BF16) return plan_single<OP_BF16, 128, 6>(stages, prev, n, kernel, num_sms, out);
        if (op == OP_I8) return plan_single<OP_I8, 128, 6>(stages, prev, n, kernel, num_sms, out);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_single_group(const GroupLaunch &g, const void *tables_dev, int *done,
                                int *status, cudaStream_t s)
{
    if (g.ctas < 1) return cudaSuccess;
    if (g.op == OP_TF32X3) return launch_single<OP_TF32X3, 128, 3>(g, tables_dev, done, status, s);
    if (g.kernel == GK_SINGLE_256) {
        if (g.op == OP_BF16) return launch_single<OP_BF16, 256, 4>(g, tables_dev, done, status, s);
        if (g.op == OP_I8) return launch_single<OP_I8, 256, 4>(g, tables_dev, done, status, s);
    } else if (g.kernel == GK_SINGLE_128) {
        if (g.op == OP_BF16) return launch_single<OP_BF16, 128, 6>(g, tables_dev, done, status, s);
        if (g.op == OP_I8) return launch_single<OP_I8, 128, 6>(g, tables_dev, done, status, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t plan_group(const StageArgs *stages, const int *prev, int n, int kernel, int num_sms,
                       GroupLaunch &out)
{
    if (n >= 1 && stages[0].op != OP_TF32X3 && kernel == GK_PAIR)
        return plan_pair_group(stages, prev, n, num_sms, out);
    return plan_single_group(stages, prev, n, kernel, num_sms, out);
}

cudaError_t launch_group(const GroupLaunch &g, const void *tables_dev, int *done, int *status,
                         cudaStream_t s)
{
    if (g.kernel == GK_PAIR && g.op != OP_TF32X3)
        return launch_pair_group(g, tables_dev, done, status, s);
    return launch_single_group(g, tables_dev, done, status, s);
}

}  // namespace fg
