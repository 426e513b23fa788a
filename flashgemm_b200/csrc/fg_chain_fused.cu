// Whole GEMM chain in one persistent launch (BF16 and INT8): the fused chain.
//
// The reference runs all stages of a 32-column panel back to back on one core
// (multigemm/src/flashgemm.c:123-148), keeping the intermediate panel in a
// per-thread buffer. Here the unit is a 256-column block: CTA pairs
// (cta_group::2, 256 x 256 tiles, as in tc_pair_kernel) walk one work list
// holding every stage's tiles, stage by stage and, inside a stage, column
// block by column block. A tile of stage i in column block n needs the whole
// of stage i-1's output in that block; when a CTA's epilogue has stored its
// part of a tile it bumps a per-(stage, block) counter, and the TMA producer
// of a stage-i tile waits for stage i-1's counter of its block to be complete
// before loading. Stage boundaries therefore cost no kernel launch and no
// wave-quantisation tail: pairs move on to the next stage's first column
// blocks while the last blocks of the previous stage finish. Intermediates
// (M_i x 256 per block, too wide for shared memory at these widths) stay in
// L2 between the two stages that touch them.
//
// Streaming hand-off (chosen per chain by the host's schedule estimate): a
// stage keeps one counter per (column block, 256-row tile) instead of one per
// column block, and the producer of the next stage waits for each row tile of
// its input only when its k-loop reaches that tile's k-blocks. With the stages'
// tiles listed row tile by row tile, a long-K stage then starts on a column
// block while the previous stage is still storing the block's last rows.
//
// Every CTA of the grid may wait on another's counters, so the grid never
// holds more pairs than the device keeps active at once (occupancy API); see
// launch_pairs for why that suffices. Every wait is bounded.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iterator>
#include <memory>
#include <mutex>
#include <type_traits>
#include <vector>

#include "fg_tc_common.cuh"

namespace fg {

constexpr int kChainMaxStages = 8;      // stage table carried in the kernel parameters
constexpr int kChainMaxPairs = 128;
constexpr int kParamSchedItems = 5632;  // work entries carried in the kernel parameters
constexpr int kParamSchedSmall = 1536;  // the same, smaller parameter blocks
constexpr int kParamSchedTiny = 512;

struct alignas(64) ChainStage {
    CUtensorMap tm_w;  // weights, M x K (box 128 rows x 128 bytes)
    CUtensorMap tm_x;  // activations, K x N (MN-major boxes)
    CUtensorMap tm_wt; // INT8 tail block (rows tail_row0 .. M-1, pre-shifted), else = tm_w
    CUtensorMap tm_out;// stage output, for the staged (TMA-store) epilogue
    StageArgs a;       // shapes and epilogue of this stage
    int tiles_m;       // pair tiles (256 rows) along M
    int tiles_n;       // 256-column blocks along N
    int prev;          // stage whose output this stage reads (-1: first stage of its chain)
    int done_off;      // this stage's counters in `done`
    int row_counters;  // 1: a counter per (column block, row tile), the reader streams;
                       // 0: a counter per column block
};

// Work entry: stage << 23 | row block << 12 | column block.
__host__ __device__ constexpr uint32_t pack_item(int stage, int mb, int nb)
{
    return ((uint32_t)stage << 23) | ((uint32_t)mb << 12) | (uint32_t)nb;
}

// Work entries are ordered so that every dependency of an entry comes earlier
// (a chain's stages in order); the host assigns entries to pairs (pair p runs
// sched[off[p] .. off[p+1]) in that order), so the earliest unfinished entry
// always heads its pair's list and the grid cannot deadlock. A single chain's
// tables travel in the kernel parameters (ChainParams, ~28 KB per launch): the
// kernel then reads its stage records and tensor maps through the constant
// cache (measured on B200 against the same tables in device memory: BF16 chain
// 67.9 against 78.4 us, INT8 chain 171.4 against 185.5 us). A grouped launch of
// many chains passes its tables in device memory (ChainParamsExt).
template <int NST, int CAP>
struct ChainParamsT {
    ChainStage st[NST];
    int npairs;
    int *done;        // per (stage, column block): epilogue warps that finished a tile
    int *status;
    unsigned long long *trace;  // optional: kTraceFields stamps per (work entry, CTA)
    int sched_off[kChainMaxPairs + 1];
    uint32_t sched[CAP];
};
using ChainParams = ChainParamsT<kChainMaxStages, kParamSchedItems>;
static_assert(sizeof(ChainParams) <= 32000, "kernel parameter space");

struct ChainParamsExt {
    const ChainStage *ext_st;
    const WorkEntry *ext_sched;
    const int *ext_off;
    int npairs;
    int *done;
    int *status;
    unsigned long long *trace;
};

template <bool EXT, int NST, int CAP> struct ChainParamsOf { using type = ChainParamsT<NST, CAP>; };
template <int NST, int CAP> struct ChainParamsOf<true, NST, CAP> { using type = ChainParamsExt; };

// Trace record of one (item, CTA): where the time of a fused chain goes.
enum { TR_ENTRY = 0, TR_SM, TR_PROD_START, TR_DEP_DONE, TR_PROD_END, TR_MMA_START, TR_MMA_END,
       TR_EPI_START, TR_EPI_ISSUED, TR_EPI_END, kTraceFields };

template <class PT>
__device__ __forceinline__ void trace_put(const PT &P, int t, uint32_t rank, int f,
                                          unsigned long long v)
{
    if (P.trace) P.trace[((size_t)t * 2 + rank) * kTraceFields + f] = v;
}


// Epilogue warps per CTA (4) x CTAs per pair (2): counter increments per tile.
constexpr int kDoneIncrementsPerTile = 8;

// Stage i and work entry q, from the parameters (read through the constant
// cache) or from device memory.
template <bool EXT, class PT>
__device__ __forceinline__ const ChainStage &stage_at(const PT &P, int i)
{
    if constexpr (EXT)
        return P.ext_st[i];
    else
        return P.st[i];
}

template <bool EXT, class PT>
__device__ __forceinline__ void entry_at(const PT &P, int q, int &si, int &mb, int &nb)
{
    if constexpr (EXT) {
        const WorkEntry e = P.ext_sched[q];
        si = (int)e.stage;
        mb = (int)(e.mbnb >> 16);
        nb = (int)(e.mbnb & 0xffffu);
    } else {
        const uint32_t e = P.sched[q];
        si = (int)(e >> 23);
        mb = (int)((e >> 12) & 2047u);
        nb = (int)(e & 4095u);
    }
}

// EXT: stage table and schedule in device memory (grouped launches) rather
// than in the parameters (single chains, read through the constant cache).
template <int OP, bool EXT, int NST = kChainMaxStages, int CAP = kParamSchedItems>
__global__ void __launch_bounds__(kThreads, 1)
    tc_chain_kernel(const __grid_constant__ typename ChainParamsOf<EXT, NST, CAP>::type P)
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
    int *status = P.status;
    int q_begin, q_end;
    if constexpr (EXT) {
        q_begin = P.ext_off[pair];
        q_end = P.ext_off[pair + 1];
    } else {
        q_begin = P.sched_off[pair];
        q_end = P.sched_off[pair + 1];
    }

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&bars->full[s], 1);
            mbar_init(&bars->empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&bars->acc_full[a], 1);
            mbar_init(&bars->acc_empty[a], 2 * 4);
        }
        mbar_init(&bars->mma_done, 1);
        bars->abort = 0;
        fence_mbar_init();
    }
    if constexpr (!EXT) {
        if (warp == 0 && lane == 0) {  // descriptors of the stages in the parameters
            for (int i = 0; i < NST; ++i)
                if (P.st[i].tiles_m) {
                    tma_prefetch_desc(&P.st[i].tm_w);
                    tma_prefetch_desc(&P.st[i].tm_x);
                    tma_prefetch_desc(&P.st[i].tm_wt);
                    tma_prefetch_desc(&P.st[i].tm_out);
                }
        }
    }
    if (warp == 1) tmem_alloc_pair(&bars->tmem_base, G::TMEM_COLS);
    tc_fence_before();
    cluster_sync();
    tc_fence_after();
    const uint32_t tmem_base = bars->tmem_base;

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer (both CTAs)
        if (lane == 0) {
            int s = 0;
            uint32_t ph = 0;
            uint32_t pending = 0, pending_ph = 0;
            for (int q = q_begin; q < q_end; ++q) {
                int si, mb, nb;
                entry_at<EXT>(P, q, si, mb, nb);
                const int t = q;
                const ChainStage &cs = stage_at<EXT>(P, si);
                const int M = cs.a.M, N = cs.a.N;
                trace_put(P, t, rank, TR_ENTRY, pack_item(si, mb, nb));
                trace_put(P, t, rank, TR_SM, smid());
                trace_put(P, t, rank, TR_PROD_START, globaltimer_ns());
                const int *row_cnt = nullptr;  // streaming: the input block's row-tile counters
                int row_tiles = 0;
                if (cs.prev >= 0 && stage_at<EXT>(P, cs.prev).row_counters) {
                    const ChainStage &ps = stage_at<EXT>(P, cs.prev);
                    row_cnt = P.done + ps.done_off + nb * ps.tiles_m;
                    row_tiles = ps.tiles_m;
                } else if (cs.prev >= 0) {
                    // the previous stage must have stored all of column block nb
                    const ChainStage &ps = stage_at<EXT>(P, cs.prev);
                    const int *cnt = P.done + ps.done_off + nb;
                    const int need = kDoneIncrementsPerTile * ps.tiles_m;
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
                    fence_proxy_async_global();
                }
                trace_put(P, t, rank, TR_DEP_DONE, globaltimer_ns());
                const int m0p = mb * G::BM;
                const int n0 = nb * BN;
                int tx = 0, my_boxes = 0;
                bool my_a = false;
                for (int r = 0; r < 2; ++r) {
                    const bool a_in = m0p + 128 * r < M;
                    int nbx = 0;
                    for (int j = 0; j < G::NBOX; ++j)
                        if (n0 + (BN / 2) * r + j * G::BOX_N < N) ++nbx;
                    tx += (a_in ? G::A_BYTES : 0) + nbx * G::BOX_BYTES;
                    if (r == (int)rank) {
                        my_a = a_in;
                        my_boxes = nbx;
                    }
                }
                // per-tile operands, kept in registers across the k-loop
                const int num_kb = (cs.a.K + G::BK - 1) / G::BK;
                const int ma = m0p + 128 * (int)rank;
                const bool a_tail = my_a && tile_has_tail(cs.a, ma);
                const CUtensorMap *tm_a = a_tail ? &cs.tm_wt : &cs.tm_w;
                const CUtensorMap *tm_b = &cs.tm_x;
                const int a_row = a_tail ? ma - cs.a.tail_row0 : ma;
                const int b_col = n0 + (BN / 2) * (int)rank;
                // k-blocks in segments: the whole K at once, or, streaming, one input
                // row tile (256 / BK k-blocks) after its counter is complete; the
                // inner loop carries no dependency check
                constexpr int kKbPerRow = 256 / G::BK;
                static_assert(256 % G::BK == 0, "k-blocks tile the 256-row input tiles");
                for (int kb0 = 0; kb0 < num_kb;) {
                    int kb1 = num_kb;
                    if (row_cnt) {
                        const int g = min(kb0 / kKbPerRow, row_tiles - 1);
                        if (ld_acquire_gpu(row_cnt + g) < kDoneIncrementsPerTile) {
                            const uint64_t t0 = globaltimer_ns();
                            while (ld_acquire_gpu(row_cnt + g) < kDoneIncrementsPerTile) {
                                __nanosleep(32);
                                if (wait_expired(t0)) {
                                    atomicCAS(status, 0, KERR_WAIT_DEPENDENCY);
                                    set_abort(bars);
                                    goto producer_done;
                                }
                            }
                        }
                        fence_proxy_async_global();
                        if (g + 1 < row_tiles) kb1 = min(num_kb, (g + 1) * kKbPerRow);
                    }
                    for (int kb = kb0; kb < kb1; ++kb) {
                        if (!mbar_wait(&bars->empty[s], ph ^ 1, status, KERR_WAIT_EMPTY)) {
                            set_abort(bars);
                            goto producer_done;
                        }
                        uint8_t *st = smem + s * G::STAGE_BYTES;
                        const uint32_t full_leader = mapa_shared(smem_u32(&bars->full[s]), 0);
                        if (leader) mbar_arrive_expect_tx(&bars->full[s], (uint32_t)tx);
                        const int k0 = kb * G::BK;
                        if (my_a) tma_load_2d_pair(st, tm_a, full_leader, k0, a_row);
                        for (int j = 0; j < my_boxes; ++j)
                            tma_load_2d_pair(st + G::A_BYTES + j * G::BOX_BYTES, tm_b, full_leader,
                                             b_col + j * G::BOX_N, k0);
                        if (leader) {
                            pending |= 1u << s;
                            pending_ph = (pending_ph & ~(1u << s)) | (ph << s);
                        }
                        if (++s == S) {
                            s = 0;
                            ph ^= 1;
                        }
                    }
                    kb0 = kb1;
                }
                trace_put(P, t, rank, TR_PROD_END, globaltimer_ns());
                if (aborted(bars)) break;
            }
        producer_done:
            for (int st = 0; st < S; ++st)
                if (pending & (1u << st))
                    mbar_wait(&bars->full[st], (pending_ph >> st) & 1u, status, KERR_WAIT_FULL);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer (leader only)
        if (lane == 0 && leader) {
            int s = 0;
            uint32_t ph = 0;
            int acc = 0;
            uint32_t acc_ph = 0;
            for (int q = q_begin; q < q_end; ++q) {
                const int t = q;
                int si, mb, nb;
                entry_at<EXT>(P, q, si, mb, nb);
                const int num_kb = (stage_at<EXT>(P, si).a.K + G::BK - 1) / G::BK;
                if (!mbar_wait(&bars->acc_empty[acc], acc_ph ^ 1, status, KERR_WAIT_ACC_EMPTY)) {
                    set_abort(bars);
                    break;
                }
                tc_fence_after();
                trace_put(P, t, rank, TR_MMA_START, globaltimer_ns());
                const uint32_t d_tmem = tmem_base + acc * BN;
                bool ok = true;
                for (int kb = 0; kb < num_kb; ++kb) {
                    if (!mbar_wait(&bars->full[s], ph, status, KERR_WAIT_FULL)) {
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
                    tc_commit_pair(&bars->empty[s], 0x3);
                    if (++s == S) {
                        s = 0;
                        ph ^= 1;
                    }
                }
                if (!ok) {
                    set_abort(bars);
                    break;
                }
                tc_commit_pair(&bars->acc_full[acc], 0x3);
                trace_put(P, t, rank, TR_MMA_END, globaltimer_ns());
                if (++acc == 2) {
                    acc = 0;
                    acc_ph ^= 1;
                }
                if (aborted(bars)) break;
            }
            tc_commit_pair(&bars->mma_done, 0x1);
            mbar_wait(&bars->mma_done, 0, status, KERR_WAIT_FULL);
        }
    } else {
        // ------------------------------------------------------------ epilogue (warps 2..5, both CTAs)
        const int quarter = warp & 3;
        int acc = 0;
        uint32_t acc_ph = 0;
        uint8_t *staging = smem + S * G::STAGE_BYTES + (warp - 2) * 2 * kStageBufBytes;
        int sbuf = 0;
        for (int q = q_begin; q < q_end; ++q) {
            int si, mb, nb;
            entry_at<EXT>(P, q, si, mb, nb);
            const int t = q;
            if (!mbar_wait(&bars->acc_full[acc], acc_ph, status, KERR_WAIT_ACC_FULL)) {
                set_abort(bars);
                break;
            }
            tc_fence_after();
            if (quarter == 0 && lane == 0) trace_put(P, t, rank, TR_EPI_START, globaltimer_ns());
            const int m0 = mb * G::BM + 128 * (int)rank;
            const int n0 = nb * BN;
            const uint32_t t_row = tmem_base + acc * BN + ((uint32_t)(quarter * 32) << 16);
            const ChainStage &cs = stage_at<EXT>(P, si);
            drain_warp<OP, BN>(cs.a, &cs.tm_out, t_row, lane, m0 + quarter * 32, n0, staging,
                               sbuf);
            tc_fence_before();
            // direct-store path: this lane's stores before the release (TMA stores
            // are ordered by lane 0's bulk wait and fences below)
            if (!cs.a.tma_store) __threadfence();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive_cluster(mapa_shared(smem_u32(&bars->acc_empty[acc]), 0));
                if (quarter == 0) trace_put(P, t, rank, TR_EPI_ISSUED, globaltimer_ns());
                // this warp's part of the tile is in memory: release it to the next stage
                bulk_wait<0>();
                fence_proxy_async_global();
                __threadfence();
                red_release_gpu_add(P.done + cs.done_off + (cs.row_counters ? nb * cs.tiles_m + mb : nb),
                                    1);
                if (quarter == 0) trace_put(P, t, rank, TR_EPI_END, globaltimer_ns());
            }
            if (++acc == 2) {
                acc = 0;
                acc_ph ^= 1;
            }
            if (aborted(bars)) break;
        }
    }

    if (warp >= 2 && lane == 0) bulk_wait<0>();
    tc_fence_before();
    __syncthreads();
    cluster_sync();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc_pair(tmem_base, G::TMEM_COLS);
    }
}

// ------------------------------------------------------------------ host side

namespace {

// Stage table entry of one stage (tensor maps, shapes, dependencies).
template <int OP>
cudaError_t make_chain_stage(const StageArgs &a, int prev, int done_off, ChainStage &cs)
{
    using T = OpTraits<OP>;
    using G = PairGeo<OP>;
    const CUtensorMapDataType dt = OP == OP_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                 : CU_TENSOR_MAP_DATA_TYPE_UINT8;
    memset(&cs, 0, sizeof cs);
    if (!make_map(&cs.tm_w, dt, T::elt, a.w, a.M, a.K, a.ld_w, G::BK, 128))
        return cudaErrorInvalidValue;
    if (!make_map(&cs.tm_x, dt, T::elt, a.x, a.K, a.N, a.ld_x, G::BOX_N, G::BK))
        return cudaErrorInvalidValue;
    if (a.tail_hi > a.tail_lo) {
        if (!make_map(&cs.tm_wt, dt, T::elt, a.w_tail, a.M - a.tail_row0, a.K, a.ld_w_tail, G::BK,
                      128))
            return cudaErrorInvalidValue;
    } else {
        cs.tm_wt = cs.tm_w;
    }
    cs.a = a;
    cs.a.tma_store = make_out_map(&cs.tm_out, cs.a) ? 1 : 0;
    if (!cs.a.tma_store) cs.tm_out = cs.tm_w;
    cs.tiles_m = (a.M + G::BM - 1) / G::BM;
    cs.tiles_n = (a.N + G::BN - 1) / G::BN;
    cs.prev = prev;
    cs.done_off = done_off;
    cs.row_counters = 0;
    if (cs.tiles_m > 65535 || cs.tiles_n > 65535) return cudaErrorNotSupported;
    return cudaSuccess;
}

// Pairs that fit on the device at once (cluster occupancy of the kernel), per device.
template <int OP>
cudaError_t pair_capacity(int num_sms, int &pairs)
{
    using G = PairGeo<OP>;
    static std::mutex mu;
    static int cap[64];
    static unsigned long long known = 0;
    std::lock_guard<std::mutex> lk(mu);
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(known & (1ull << (dev & 63)))) {
        cudaError_t e = cudaFuncSetAttribute(tc_chain_kernel<OP, false>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM_BYTES);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(tc_chain_kernel<OP, true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM_BYTES);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(tc_chain_kernel<OP, false, 8, kParamSchedSmall>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM_BYTES);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(tc_chain_kernel<OP, false, 4, kParamSchedSmall>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM_BYTES);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(tc_chain_kernel<OP, false, 4, kParamSchedTiny>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 2;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.blockDim = dim3(kThreads);
        cfg.dynamicSmemBytes = G::SMEM_BYTES;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int dev_sms = 0;
        cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, dev);
        cfg.gridDim = dim3(2 * (dev_sms / 2));
        int clusters = 0;
        e = cudaOccupancyMaxActiveClusters(&clusters, tc_chain_kernel<OP, false>, &cfg);
        if (e != cudaSuccess || clusters < 1) {
            cudaGetLastError();
            return cudaErrorNotSupported;
        }
        cap[dev & 63] = clusters < kChainMaxPairs ? clusters : kChainMaxPairs;
        known |= 1ull << (dev & 63);
    }
    pairs = cap[dev & 63];
    if (pairs > num_sms / 2) pairs = num_sms / 2 > 0 ? num_sms / 2 : 1;  // a cap below the device
    return cudaSuccess;
}

template <int OP, bool EXT, int NST = kChainMaxStages, int CAP = kParamSchedItems>
cudaError_t launch_pairs(const typename ChainParamsOf<EXT, NST, CAP>::type &P, int pairs,
                         cudaStream_t s)
{
    using G = PairGeo<OP>;
    // Pairs wait on one another, so all must become resident: `pairs` never
    // exceeds the device's maximum of active clusters for this kernel (occupancy
    // API), and a pair only ever waits on pairs of its own grid, which run to
    // completion once resident; pairs held back behind another kernel's CTAs
    // start when that kernel ends. Every wait is bounded in any case. (No
    // cooperative flag: cluster launches with it cannot be profiled.)
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
    cfg.gridDim = dim3(2 * pairs);
    return cudaLaunchKernelEx(&cfg, tc_chain_kernel<OP, EXT, NST, CAP>, P);
}

// Schedule model in k-block units (a tile costs its k-blocks plus 6 for the
// epilogue and hand-off). Streaming (row_counters): the stages' tiles are listed
// row tile by row tile, and a reading stage's tile needs input row tile g only
// after its first g * 256 / bk k-blocks.
std::vector<SchedStage> sched_stages(const std::vector<ChainStage> &st, int bk)
{
    std::vector<SchedStage> ss(st.size());
    for (size_t i = 0; i < st.size(); ++i) {
        ss[i] = SchedStage{st[i].tiles_m, st[i].tiles_n, st[i].prev, st[i].done_off,
                           (double)((st[i].a.K + bk - 1) / bk) + 6.0};
        const bool streamed = st[i].prev >= 0 && st[st[i].prev].row_counters;
        ss[i].row_done = st[i].row_counters;
        ss[i].row_major = st[i].row_counters || streamed;
        ss[i].stream = streamed ? 256.0 / bk : 0.0;
    }
    return ss;
}

// Counter layout of a chain: bit i of `stream` gives stage i (not the last) a
// counter per (column block, row tile), so that stage i + 1 streams.
void set_counters(std::vector<ChainStage> &st, unsigned stream)
{
    int done_off = 0;
    const int n = (int)st.size();
    for (int i = 0; i < n; ++i) {
        st[i].row_counters = ((stream >> i) & 1u) && i + 1 < n ? 1 : 0;
        st[i].done_off = done_off;
        done_off += st[i].tiles_n * (st[i].row_counters ? st[i].tiles_m : 1);
    }
}

// FG_CHAIN_STREAM: 0 = never stream, 1 = every stage boundary, m<bits> = the
// boundaries whose bits are set (bit i: stage i + 1 streams from stage i),
// unset = every boundary when the schedule estimate is at least 1 % shorter,
// else none. (Measured on B200: the BF16 chain 4096x1024 -> 4096 -> 1024 ->
// 1024, estimate 0.978 of block-wise, ran 4 % faster streamed; the INT8 chain
// 8192x2048 -> 4096 -> 2048 -> 4096 -> 1024, estimate 1.008, 15 % slower.)
// FG_CHAIN_WINDOW=<blocks>: place a single chain's tiles that many 256-column
// blocks at a time, every stage of them before the next blocks' (SchedOpts);
// unset or 0: each stage whole.
int window_blocks()
{
    static const int w = [] {
        const char *v = getenv("FG_CHAIN_WINDOW");
        return v ? atoi(v) : 0;
    }();
    return w > 0 ? w : 0;
}

// FG_CHAIN_FEED=0: no feeder workers (see SchedOpts) in a single chain's schedule;
// FG_CHAIN_FEED=<stage>,<pairs>,<rows>: exactly those feeders (when that stage's
// boundary streams); otherwise the host tries them at every streamed boundary and
// keeps them when the estimate is at least 1 % shorter.
bool feed_mode()
{
    static const bool on = [] {
        const char *v = getenv("FG_CHAIN_FEED");
        return !(v && v[0] == '0' && v[1] == 0);
    }();
    return on;
}
bool feed_forced(SchedOpts &o)
{
    static const int f[3] = {-1, 0, 0};
    static const bool forced = [] {
        const char *v = getenv("FG_CHAIN_FEED");
        int a = -1, b = 0, c = 0;
        if (v && sscanf(v, "%d,%d,%d", &a, &b, &c) == 3 && a >= 0 && b > 0 && c > 0) {
            const_cast<int *>(f)[0] = a;
            const_cast<int *>(f)[1] = b;
            const_cast<int *>(f)[2] = c;
            return true;
        }
        return false;
    }();
    if (!forced) return false;
    o.feed_stage = f[0];
    o.feed_workers = f[1];
    o.feed_rows = f[2];
    return true;
}

// FG_CHAIN_PARAMS=big: every single chain launches with the largest parameter
// block (28 KB); otherwise with the smallest one its stages and schedule fit
// (measured on B200: BF16 chain 4096 x 1024 -> 4096 -> 1024 -> 1024, 3 stages
// and 384 entries, 66.5 us per launch with the 5 KB block against 68.0 with the
// 28 KB one; INT8 chain 8192 x 2048 -> 4096 -> 2048 -> 4096 -> 1024, 4 stages
// and 1408 entries, 168.8 against 170.5 us with the 9 KB block).
bool big_params()
{
    static const bool big = [] {
        const char *v = getenv("FG_CHAIN_PARAMS");
        return v && strcmp(v, "big") == 0;
    }();
    return big;
}

constexpr unsigned kStreamAuto = ~0u;
unsigned stream_mode()
{
    static const unsigned m = [] {
        const char *v = getenv("FG_CHAIN_STREAM");
        if (!v) return kStreamAuto;
        if (v[0] == 'm') return (unsigned)strtoul(v + 1, nullptr, 10) & 0xffu;
        return v[0] == '1' ? 0xffu : 0u;
    }();
    return m;
}

}  // namespace

// Everything a chain's launch parameters depend on besides the counters and the
// trace buffer: the stages' operands, shapes and epilogues, the grid, the mode.
static std::vector<long> params_key(const StageArgs *st, int n, int device, int num_sms)
{
    std::vector<long> k = {device, num_sms, n, (long)stream_mode()};
    for (int i = 0; i < n; ++i) {
        const StageArgs &a = st[i];
        const long v[] = {a.op, a.M, a.N, a.K, (long)a.w, (long)a.w_lo, a.ld_w, (long)a.x,
                          (long)a.x_lo, a.ld_x, a.epi, (long)a.out, (long)a.out_lo, a.ld_out,
                          a.permute, a.m_written, a.tail_lo, a.tail_hi, (long)a.w_tail,
                          a.ld_w_tail, a.tail_row0, a.kchunk, (long)a.status};
        k.insert(k.end(), std::begin(v), std::end(v));
    }
    return k;
}

// One chain (stage i reads stage i - 1) with its tables in the kernel parameters.
// A launch with the same operands and shapes as one of the last few reuses its
// parameter block (tensor maps, stage table, schedule), changing only the
// counters and the trace buffer.
template <int OP>
static cudaError_t launch_chain_op(const StageArgs *stages, int n, int *done, int *status,
                                   unsigned long long *trace, int num_sms, cudaStream_t s)
{
    using G = PairGeo<OP>;
    if (n > kChainMaxStages) return cudaErrorNotSupported;
    static std::mutex mu;  // parameter blocks (~28 KB each) are shared: one launch at a time
    std::lock_guard<std::mutex> lk(mu);
    struct Built {
        std::vector<long> key;
        ChainParams P;
        // the same tables in the smallest parameter block they fit (less to copy
        // into the constant bank per launch): 4 stages x 512 entries, 4 x 1536,
        // 8 x 1536, else P itself
        int form = 0;
        std::unique_ptr<ChainParamsT<4, kParamSchedTiny>> s4t;
        std::unique_ptr<ChainParamsT<4, kParamSchedSmall>> s4s;
        std::unique_ptr<ChainParamsT<8, kParamSchedSmall>> s8s;
    };
    auto launch_built = [&](Built *b) -> cudaError_t {
        switch (b->form) {
        case 1: return launch_pairs<OP, false, 4, kParamSchedTiny>(*b->s4t, b->P.npairs, s);
        case 2: return launch_pairs<OP, false, 4, kParamSchedSmall>(*b->s4s, b->P.npairs, s);
        case 3: return launch_pairs<OP, false, 8, kParamSchedSmall>(*b->s8s, b->P.npairs, s);
        default: return launch_pairs<OP, false>(b->P, b->P.npairs, s);
        }
    };
    auto set_run = [](Built *b, int *done, int *status, unsigned long long *trace) {
        auto set = [&](auto *q) {
            if (!q) return;
            q->done = done;
            q->status = status;
            q->trace = trace;
        };
        set(&b->P);
        set(b->s4t.get());
        set(b->s4s.get());
        set(b->s8s.get());
    };
    static std::vector<Built *> built;  // most recently used last, at most kBuiltKept
    constexpr size_t kBuiltKept = 8;
    int device = 0;
    cudaGetDevice(&device);
    std::vector<long> pkey = params_key(stages, n, device, num_sms);
    for (size_t j = 0; j < built.size(); ++j)
        if (built[j]->key == pkey) {
            Built *b = built[j];
            built.erase(built.begin() + j);
            built.push_back(b);
            set_run(b, done, status, trace);
            return launch_built(b);
        }
    std::unique_ptr<Built> slot;  // back into `built` once complete; freed on an early return
    if (built.size() >= kBuiltKept) {
        slot.reset(built.front());
        built.erase(built.begin());
    } else {
        slot.reset(new Built);
    }
    slot->key.clear();
    slot->form = 0;
    slot->s4t.reset();
    slot->s4s.reset();
    slot->s8s.reset();
    ChainParams &P = slot->P;
    memset(&P, 0, sizeof P);
    std::vector<ChainStage> st(n);
    long items = 0;
    for (int i = 0; i < n; ++i) {
        cudaError_t e = make_chain_stage<OP>(stages[i], i - 1, 0, st[i]);
        if (e != cudaSuccess) return e;
        if (st[i].tiles_m > 2047 || st[i].tiles_n > 4095) return cudaErrorNotSupported;
        items += (long)st[i].tiles_m * st[i].tiles_n;
    }
    if (items > kParamSchedItems) return cudaErrorNotSupported;
    int pairs = 0;
    cudaError_t e = pair_capacity<OP>(num_sms, pairs);
    if (e != cudaSuccess) return e;
    if (items < pairs) pairs = (int)items;
    P.npairs = pairs;
    P.done = done;
    P.status = status;
    P.trace = trace;

    // the schedule depends only on the shapes: computed once per shape set
    struct Cached {
        std::vector<long> key;
        unsigned stream;  // stage boundaries that stream
        SchedOpts opts;   // feeders and window of the chosen schedule
        std::vector<int> off;
        std::vector<uint32_t> items;
    };
    static std::vector<Cached> cache;
    std::vector<long> key = {pairs, n};
    for (int i = 0; i < n; ++i) {
        key.push_back(stages[i].M);
        key.push_back(stages[i].K);
        key.push_back(stages[i].N);
    }
    const Cached *sc = nullptr;
    for (const Cached &c : cache)
        if (c.key == key) sc = &c;
    if (!sc) {
        Cached c;
        c.key = key;
        std::vector<WorkEntry> ent;
        // block-wise or streaming hand-off, whichever the estimate prefers
        double span_block = 0.0, span_stream = 0.0;
        std::vector<int> off_s;
        std::vector<WorkEntry> ent_s;
        SchedOpts base;
        base.window = window_blocks();
        c.opts = base;
        set_counters(st, 0u);
        list_schedule(sched_stages(st, G::BK).data(), n, pairs, 2.0, c.off, ent, &span_block,
                      nullptr, &base);
        c.stream = 0u;
        const unsigned mode = stream_mode();
        if (n > 1 && mode != 0u) {
            const unsigned mask = mode == kStreamAuto ? 0xffu : mode;
            set_counters(st, mask);
            const std::vector<SchedStage> ss = sched_stages(st, G::BK);
            list_schedule(ss.data(), n, pairs, 2.0, off_s, ent_s, &span_stream, nullptr, &base);
            // feeders at a streamed boundary (see SchedOpts): the best of a small grid
            SchedOpts chosen = base;
            SchedOpts forced = base;
            if (feed_forced(forced) && forced.feed_stage + 1 < n && ((mask >> forced.feed_stage) & 1u)) {
                list_schedule(ss.data(), n, pairs, 2.0, off_s, ent_s, &span_stream, nullptr, &forced);
                chosen = forced;
            } else if (feed_mode()) {
                SchedOpts best = base;
                double span_best = span_stream;
                std::vector<int> off_f;
                std::vector<WorkEntry> ent_f;
                for (int f = 0; f + 1 < n; ++f) {
                    if (!((mask >> f) & 1u)) continue;
                    for (int q = 2; q <= pairs / 4; q += 2)
                        for (int d = 1; d <= std::min(8, st[f].tiles_m - 1); ++d) {
                            SchedOpts fd = base;
                            fd.feed_stage = f;
                            fd.feed_workers = q;
                            fd.feed_rows = d;
                            double span_f = 0.0;
                            list_schedule(ss.data(), n, pairs, 2.0, off_f, ent_f, &span_f, nullptr, &fd);
                            if (span_f < span_best - 1e-9) span_best = span_f, best = fd;
                        }
                }
                if (best.feed_stage >= 0 && span_best < 0.99 * span_stream) {
                    list_schedule(ss.data(), n, pairs, 2.0, off_s, ent_s, &span_stream, nullptr, &best);
                    chosen = best;
                }
            }
            if (mode != kStreamAuto || span_stream < 0.99 * span_block) {
                c.stream = mask;
                c.opts = chosen;
                c.off.swap(off_s);
                ent.swap(ent_s);
            }
        }
        for (const WorkEntry &w : ent)
            c.items.push_back(pack_item((int)w.stage, (int)(w.mbnb >> 16), (int)(w.mbnb & 0xffffu)));
        if (cache.size() >= 32) cache.erase(cache.begin());
        cache.push_back(std::move(c));
        sc = &cache.back();
    }
    set_counters(st, sc->stream);
    for (int i = 0; i < n; ++i) P.st[i] = st[i];
    for (int p = 0; p <= pairs; ++p) P.sched_off[p] = sc->off[p];
    memcpy(P.sched, sc->items.data(), sc->items.size() * sizeof(uint32_t));
    const size_t nitems = sc->items.size();
    auto shrink = [&](auto &dst) {
        using PT = typename std::remove_reference<decltype(*dst)>::type;
        dst.reset(new PT);
        memset(dst.get(), 0, sizeof(PT));
        for (int i = 0; i < n; ++i) dst->st[i] = P.st[i];
        dst->npairs = P.npairs;
        dst->done = P.done;
        dst->status = P.status;
        dst->trace = P.trace;
        memcpy(dst->sched_off, P.sched_off, sizeof dst->sched_off);
        memcpy(dst->sched, P.sched, nitems * sizeof(uint32_t));
    };
    if (!big_params()) {
        if (n <= 4 && nitems <= (size_t)kParamSchedTiny) {
            shrink(slot->s4t);
            slot->form = 1;
        } else if (n <= 4 && nitems <= (size_t)kParamSchedSmall) {
            shrink(slot->s4s);
            slot->form = 2;
        } else if (nitems <= (size_t)kParamSchedSmall) {
            shrink(slot->s8s);
            slot->form = 3;
        }
    }
    slot->key.swap(pkey);
    Built *b = slot.release();
    built.push_back(b);
    return launch_built(b);
}

// Time-out self-test: a BF16 chain of two stages whose second stage waits on
// column-block counters that no tile releases (those of a third, unlisted copy
// of the first stage), with every wait of this launch limited to limit_ns.
// The second stage's producers, its MMA issuer and its epilogue warps run out,
// record an error code in *status, stop and return; the first stage's tiles
// complete. The limit is set and restored in stream order around the launch.
// `done` holds 3 * chain_counter_ints zeroed ints.
cudaError_t launch_tc_chain_stuck(const StageArgs *stages, int *done, int *status, int num_sms,
                                  unsigned long long limit_ns, cudaStream_t s)
{
    using G = PairGeo<OP_BF16>;
    if (stages[0].op != OP_BF16 || stages[1].op != OP_BF16) return cudaErrorInvalidValue;
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    std::unique_ptr<ChainParams> P(new ChainParams);
    memset(P.get(), 0, sizeof *P);
    std::vector<ChainStage> st(2);
    for (int i = 0; i < 2; ++i) {
        cudaError_t e = make_chain_stage<OP_BF16>(stages[i], i - 1, 0, st[i]);
        if (e != cudaSuccess) return e;
    }
    set_counters(st, 0u);
    int pairs = 0;
    cudaError_t e = pair_capacity<OP_BF16>(num_sms, pairs);
    if (e != cudaSuccess) return e;
    const long items = (long)st[0].tiles_m * st[0].tiles_n + (long)st[1].tiles_m * st[1].tiles_n;
    if (items > kParamSchedItems) return cudaErrorNotSupported;
    if (items < pairs) pairs = (int)items;
    std::vector<int> off;
    std::vector<WorkEntry> ent;
    list_schedule(sched_stages(st, G::BK).data(), 2, pairs, 2.0, off, ent);
    P->st[0] = st[0];
    P->st[1] = st[1];
    P->st[2] = st[0];  // never listed: its counters are never released
    P->st[2].done_off = st[1].done_off + st[1].tiles_n;
    P->st[1].prev = 2;
    P->npairs = pairs;
    P->done = done;
    P->status = status;
    for (int p = 0; p <= pairs; ++p) P->sched_off[p] = off[p];
    for (size_t i = 0; i < ent.size(); ++i)
        P->sched[i] = pack_item((int)ent[i].stage, (int)(ent[i].mbnb >> 16), (int)(ent[i].mbnb & 0xffffu));
    static const unsigned long long dflt = kWaitLimitNs;
    static unsigned long long lowered;
    lowered = limit_ns;
    e = cudaMemcpyToSymbolAsync(fg_wait_limit_ns, &lowered, sizeof lowered, 0,
                                cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    e = launch_pairs<OP_BF16, false>(*P, pairs, s);
    const cudaError_t e2 = cudaMemcpyToSymbolAsync(fg_wait_limit_ns, &dflt, sizeof dflt, 0,
                                                   cudaMemcpyHostToDevice, s);
    return e != cudaSuccess ? e : e2;
}

cudaError_t launch_tc_chain(const StageArgs *stages, int n, int *done, int *status,
                            unsigned long long *trace, int num_sms, cudaStream_t s)
{
    if (n < 1) return cudaErrorInvalidValue;
    for (int i = 0; i < n; ++i)
        if (stages[i].op != stages[0].op || stages[i].M <= 0 || stages[i].K <= 0 ||
            stages[i].N <= 0)
            return cudaErrorInvalidValue;
    switch (stages[0].op) {
    case OP_BF16: return launch_chain_op<OP_BF16>(stages, n, done, status, trace, num_sms, s);
    case OP_I8: return launch_chain_op<OP_I8>(stages, n, done, status, trace, num_sms, s);
    default: return cudaErrorInvalidValue;
    }
}

// Many stages with their tables in device memory.
template <int OP>
static cudaError_t plan_pair_op(const StageArgs *stages, const int *prev, int n, int num_sms,
                                GroupLaunch &out)
{
    using G = PairGeo<OP>;
    std::vector<ChainStage> st(n);
    long items = 0;
    int done_off = 0;
    for (int i = 0; i < n; ++i) {
        if (prev[i] >= i) return cudaErrorInvalidValue;
        cudaError_t e = make_chain_stage<OP>(stages[i], prev[i], done_off, st[i]);
        if (e != cudaSuccess) return e;
        done_off += st[i].tiles_n;
        items += (long)st[i].tiles_m * st[i].tiles_n;
    }
    int pairs = 0;
    cudaError_t e = pair_capacity<OP>(num_sms, pairs);
    if (e != cudaSuccess) return e;
    if (items < pairs) pairs = (int)items;
    std::vector<int> off;
    std::vector<WorkEntry> ent;
    const std::vector<SchedStage> ss = sched_stages(st, G::BK);
    list_schedule(ss.data(), n, pairs, 2.0, off, ent);
    auto r = [](size_t b) { return (b + 255) & ~(size_t)255; };
    out.kernel = GK_PAIR;
    out.op = OP;
    out.ctas = 2 * pairs;
    out.entries = items;
    out.done_ints = (size_t)done_off;
    out.off_st = 0;
    out.off_sched = r((size_t)n * sizeof(ChainStage));
    out.off_off = out.off_sched + r((size_t)items * sizeof(WorkEntry));
    out.tables.assign(out.off_off + r((size_t)(pairs + 1) * sizeof(int)), 0);
    memcpy(out.tables.data(), st.data(), (size_t)n * sizeof(ChainStage));
    memcpy(out.tables.data() + out.off_sched, ent.data(), (size_t)items * sizeof(WorkEntry));
    memcpy(out.tables.data() + out.off_off, off.data(), (size_t)(pairs + 1) * sizeof(int));
    return cudaSuccess;
}

cudaError_t plan_pair_group(const StageArgs *stages, const int *prev, int n, int num_sms,
                            GroupLaunch &out)
{
    if (n < 1) return cudaErrorInvalidValue;
    for (int i = 0; i < n; ++i)
        if (stages[i].op != stages[0].op || stages[i].M <= 0 || stages[i].K <= 0 ||
            stages[i].N <= 0)
            return cudaErrorInvalidValue;
    switch (stages[0].op) {
    case OP_BF16: return plan_pair_op<OP_BF16>(stages, prev, n, num_sms, out);
    case OP_I8: return plan_pair_op<OP_I8>(stages, prev, n, num_sms, out);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_pair_group(const GroupLaunch &g, const void *tables_dev, int *done,
                              int *status, cudaStream_t s)
{
    ChainParamsExt P;
    P.ext_st = reinterpret_cast<const ChainStage *>(static_cast<const unsigned char *>(tables_dev) +
                                                    g.off_st);
    P.ext_sched = reinterpret_cast<const WorkEntry *>(
        static_cast<const unsigned char *>(tables_dev) + g.off_sched);
    P.ext_off = reinterpret_cast<const int *>(static_cast<const unsigned char *>(tables_dev) +
                                              g.off_off);
    P.npairs = g.ctas / 2;
    P.done = done;
    P.status = status;
    P.trace = nullptr;
    switch (g.op) {
    case OP_BF16: return launch_pairs<OP_BF16, true>(P, g.ctas / 2, s);
    case OP_I8: return launch_pairs<OP_I8, true>(P, g.ctas / 2, s);
    default: return cudaErrorInvalidValue;
    }
}

int chain_max_stages() { return kChainMaxStages; }

size_t chain_counter_ints(int n, const long *M, long N)
{
    size_t c = 0;
    for (int i = 0; i < n; ++i) c += (size_t)((M[i] + 255) / 256) * (size_t)((N + 255) / 256);
    return c;
}
int chain_trace_fields() { return kTraceFields; }

}  // namespace fg
