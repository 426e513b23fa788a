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
// Every CTA of the grid may wait on another's counters, so the kernel is
// launched cooperatively (all CTAs co-resident, or the launch fails and the
// caller falls back to one launch per stage). Every wait is bounded.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "fg_tc_common.cuh"

namespace fg {

constexpr int kChainMaxStages = 8;
constexpr int kChainMaxPairs = 128;
constexpr int kChainMaxItems = 10240;  // schedule entries carried in the kernel parameters

struct alignas(64) ChainStage {
    CUtensorMap tm_w;  // weights, M x K (box 128 rows x 128 bytes)
    CUtensorMap tm_x;  // activations, K x N (MN-major boxes)
    CUtensorMap tm_wt; // INT8 tail block (rows tail_row0 .. M-1, pre-shifted), else = tm_w
    CUtensorMap tm_out;// stage output, for the staged (TMA-store) epilogue
    StageArgs a;       // shapes and epilogue of this stage
    int tiles_m;       // pair tiles (256 rows) along M
    int item0;         // first work item of this stage
};

// Work items are numbered stage by stage, column block by column block, row
// block by row block; every dependency of an item has a smaller number. The
// host assigns items to pairs (sched_off / sched: pair p runs items
// sched[sched_off[p] .. sched_off[p+1]) in increasing order), so the smallest
// unfinished item always heads its pair's list and the grid cannot deadlock.
struct ChainParams {
    ChainStage st[kChainMaxStages];
    int nstages;
    int tiles_n;      // 256-column blocks
    int total_items;
    int npairs;
    int *done;        // [nstages][tiles_n]: epilogue warps that finished a tile of the block
    int *status;
    unsigned long long *trace;  // optional: kTraceFields %globaltimer stamps per (item, CTA)
    uint16_t sched_off[kChainMaxPairs + 1];
    uint16_t sched[kChainMaxItems];
};

__device__ __forceinline__ int ld_acquire_gpu(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void red_release_gpu_add(int *p, int v)
{
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Generic-proxy writes / reads of global memory ordered with async-proxy (TMA) accesses.
__device__ __forceinline__ void fence_proxy_async_global()
{
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void decode_item(const ChainParams &P, int t, int &stage, int &mb,
                                            int &nb)
{
    stage = 0;
    while (stage + 1 < P.nstages && t >= P.st[stage + 1].item0) ++stage;
    const int u = t - P.st[stage].item0;
    nb = u / P.st[stage].tiles_m;
    mb = u - nb * P.st[stage].tiles_m;
}

// Trace record of one (item, CTA): where the time of a fused chain goes.
enum { TR_SM = 0, TR_PROD_START, TR_DEP_DONE, TR_PROD_END, TR_MMA_START, TR_MMA_END, TR_EPI_START,
       TR_EPI_ISSUED, TR_EPI_END, kTraceFields };

__device__ __forceinline__ void trace_put(const ChainParams &P, int t, uint32_t rank, int f,
                                          unsigned long long v)
{
    if (P.trace) P.trace[((size_t)t * 2 + rank) * kTraceFields + f] = v;
}

__device__ __forceinline__ uint32_t smid()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(r));
    return r;
}

// Epilogue warps per CTA (4) x CTAs per pair (2): counter increments per tile.
constexpr int kDoneIncrementsPerTile = 8;

template <int OP>
__global__ void __launch_bounds__(kThreads, 1) tc_chain_kernel(const __grid_constant__ ChainParams P)
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
    if (warp == 0 && lane == 0) {
        for (int i = 0; i < P.nstages; ++i) {
            tma_prefetch_desc(&P.st[i].tm_w);
            tma_prefetch_desc(&P.st[i].tm_x);
            tma_prefetch_desc(&P.st[i].tm_wt);
            tma_prefetch_desc(&P.st[i].tm_out);
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
            for (int q = P.sched_off[pair]; q < P.sched_off[pair + 1]; ++q) {
                const int t = P.sched[q];
                int si, mb, nb;
                decode_item(P, t, si, mb, nb);
                const ChainStage &cs = P.st[si];
                const int M = cs.a.M, N = cs.a.N;
                trace_put(P, t, rank, TR_SM, smid());
                trace_put(P, t, rank, TR_PROD_START, globaltimer_ns());
                if (si > 0) {
                    // stage si-1 must have stored all of column block nb
                    const int *cnt = P.done + (si - 1) * P.tiles_n + nb;
                    const int need = kDoneIncrementsPerTile * P.st[si - 1].tiles_m;
                    if (ld_acquire_gpu(cnt) < need) {
                        const uint64_t t0 = globaltimer_ns();
                        while (ld_acquire_gpu(cnt) < need) {
                            __nanosleep(64);
                            if (globaltimer_ns() - t0 > kWaitLimitNs) {
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
                const int num_kb = (cs.a.K + G::BK - 1) / G::BK;
                for (int kb = 0; kb < num_kb; ++kb) {
                    if (!mbar_wait(&bars->empty[s], ph ^ 1, status, KERR_WAIT_EMPTY)) {
                        set_abort(bars);
                        goto producer_done;
                    }
                    uint8_t *st = smem + s * G::STAGE_BYTES;
                    const uint32_t full_leader = mapa_shared(smem_u32(&bars->full[s]), 0);
                    if (leader) mbar_arrive_expect_tx(&bars->full[s], (uint32_t)tx);
                    const int k0 = kb * G::BK;
                    if (my_a) {
                        const int ma = m0p + 128 * (int)rank;
                        if (tile_has_tail(cs.a, ma))
                            tma_load_2d_pair(st, &cs.tm_wt, full_leader, k0, ma - cs.a.tail_row0);
                        else
                            tma_load_2d_pair(st, &cs.tm_w, full_leader, k0, ma);
                    }
                    for (int j = 0; j < my_boxes; ++j)
                        tma_load_2d_pair(st + G::A_BYTES + j * G::BOX_BYTES, &cs.tm_x, full_leader,
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
            for (int q = P.sched_off[pair]; q < P.sched_off[pair + 1]; ++q) {
                const int t = P.sched[q];
                int si, mb, nb;
                decode_item(P, t, si, mb, nb);
                const int num_kb = (P.st[si].a.K + G::BK - 1) / G::BK;
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
        for (int q = P.sched_off[pair]; q < P.sched_off[pair + 1]; ++q) {
            const int t = P.sched[q];
            int si, mb, nb;
            decode_item(P, t, si, mb, nb);
            if (!mbar_wait(&bars->acc_full[acc], acc_ph, status, KERR_WAIT_ACC_FULL)) {
                set_abort(bars);
                break;
            }
            tc_fence_after();
            if (quarter == 0 && lane == 0) trace_put(P, t, rank, TR_EPI_START, globaltimer_ns());
            const int m0 = mb * G::BM + 128 * (int)rank;
            const int n0 = nb * BN;
            const uint32_t t_row = tmem_base + acc * BN + ((uint32_t)(quarter * 32) << 16);
            drain_warp<OP, BN>(P.st[si].a, &P.st[si].tm_out, t_row, lane, m0 + quarter * 32, n0,
                               staging, sbuf);
            tc_fence_before();
            __threadfence();  // direct-store path: this lane's stores before the release
            __syncwarp();
            if (lane == 0) {
                mbar_arrive_cluster(mapa_shared(smem_u32(&bars->acc_empty[acc]), 0));
                if (quarter == 0) trace_put(P, t, rank, TR_EPI_ISSUED, globaltimer_ns());
                // this warp's part of the tile is in memory: release it to the next stage
                bulk_wait<0>();
                fence_proxy_async_global();
                __threadfence();
                red_release_gpu_add(P.done + si * P.tiles_n + nb, 1);
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

template <int OP>
static cudaError_t launch_chain_op(const StageArgs *stages, int n, int *done, int *status,
                                   unsigned long long *trace, int num_sms, cudaStream_t s)
{
    using T = OpTraits<OP>;
    using G = PairGeo<OP>;
    static std::mutex mu;  // P and the schedule scratch are static (~28 KB): one launch at a time
    std::lock_guard<std::mutex> lk(mu);
    static ChainParams P;
    memset(&P, 0, sizeof P);
    CUtensorMapDataType dt = OP == OP_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                           : CU_TENSOR_MAP_DATA_TYPE_UINT8;
    const int N = stages[0].N;
    P.nstages = n;
    P.tiles_n = (N + G::BN - 1) / G::BN;
    P.done = done;
    P.status = status;
    P.trace = trace;
    int items = 0;
    for (int i = 0; i < n; ++i) {
        const StageArgs &a = stages[i];
        ChainStage &cs = P.st[i];
        if (!make_map(&cs.tm_w, dt, T::elt, a.w, a.M, a.K, a.ld_w, G::BK, 128))
            return cudaErrorInvalidValue;
        if (!make_map(&cs.tm_x, dt, T::elt, a.x, a.K, a.N, a.ld_x, G::BOX_N, G::BK))
            return cudaErrorInvalidValue;
        if (a.tail_hi > a.tail_lo) {
            if (!make_map(&cs.tm_wt, dt, T::elt, a.w_tail, a.M - a.tail_row0, a.K, a.ld_w_tail,
                          G::BK, 128))
                return cudaErrorInvalidValue;
        } else {
            cs.tm_wt = cs.tm_w;
        }
        cs.a = a;
        cs.a.tma_store = make_out_map(&cs.tm_out, cs.a) ? 1 : 0;
        if (!cs.a.tma_store) cs.tm_out = cs.tm_w;
        cs.tiles_m = (a.M + G::BM - 1) / G::BM;
        cs.item0 = items;
        items += cs.tiles_m * P.tiles_n;
    }
    P.total_items = items;
    if (items > kChainMaxItems) return cudaErrorNotSupported;

    static unsigned long long attr_set = 0;
    static int max_pairs[64];
    int dev = 0;
    cudaGetDevice(&dev);
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeCooperative;
    attr[1].val.cooperative = 1;
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = G::SMEM_BYTES;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;  // occupancy query without the cooperative flag
    if (!(attr_set & (1ull << (dev & 63)))) {
        cudaError_t e = cudaFuncSetAttribute(tc_chain_kernel<OP>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM_BYTES);
        if (e != cudaSuccess) return e;
        int clusters = 0;
        cfg.gridDim = dim3(2 * (num_sms / 2));
        e = cudaOccupancyMaxActiveClusters(&clusters, tc_chain_kernel<OP>, &cfg);
        if (e != cudaSuccess || clusters < 1) {
            cudaGetLastError();
            return cudaErrorNotSupported;
        }
        max_pairs[dev & 63] = clusters;
        attr_set |= 1ull << (dev & 63);
    }
    int pairs = items < max_pairs[dev & 63] ? items : max_pairs[dev & 63];
    if (pairs > kChainMaxPairs) pairs = kChainMaxPairs;
    P.npairs = pairs;
    // The schedule depends only on the shapes: computed once per shape set.
    struct Sched {
        std::vector<long> key;
        std::vector<uint16_t> off, items;
    };
    static std::vector<Sched> cache;
    std::vector<long> key = {pairs, n, N};
    for (int i = 0; i < n; ++i) {
        key.push_back(stages[i].M);
        key.push_back(stages[i].K);
    }
    for (const Sched &c : cache)
        if (c.key == key) {
            memcpy(P.sched_off, c.off.data(), c.off.size() * sizeof(uint16_t));
            memcpy(P.sched, c.items.data(), c.items.size() * sizeof(uint16_t));
            cfg.gridDim = dim3(2 * pairs);
            cfg.numAttrs = 2;
            return cudaLaunchKernelEx(&cfg, tc_chain_kernel<OP>, P);
        }
    // List schedule in item order with estimated times: an item can start when
    // its pair is free and the previous stage's tiles of its column block have
    // finished; it goes to the pair that can start it first. Cost model: k-blocks
    // of MMA plus a fixed per-tile epilogue / hand-off overhead (both in units
    // of one k-block).
    {
        static double pair_free[kChainMaxPairs];
        static double fin[kChainMaxItems];
        static int owner[kChainMaxItems];
        static double block_done[kChainMaxStages][1024];
        int count[kChainMaxPairs];
        const int tn = P.tiles_n < 1024 ? P.tiles_n : 1024;
        for (int p = 0; p < pairs; ++p) pair_free[p] = 0.0, count[p] = 0;
        for (int i = 0; i < n; ++i)
            for (int b = 0; b < tn; ++b) block_done[i][b] = 0.0;
        for (int t = 0; t < items; ++t) {
            int si = 0;
            while (si + 1 < n && t >= P.st[si + 1].item0) ++si;
            const int u = t - P.st[si].item0;
            const int nb = u / P.st[si].tiles_m;
            const double cost = (double)((P.st[si].a.K + G::BK - 1) / G::BK) + 6.0;
            const double ready = (si > 0 && nb < tn) ? block_done[si - 1][nb] + 2.0 : 0.0;
            int best = 0;
            double best_start = 1e300;
            for (int p = 0; p < pairs; ++p) {
                const double st = pair_free[p] > ready ? pair_free[p] : ready;
                if (st < best_start - 1e-9) best_start = st, best = p;
            }
            fin[t] = best_start + cost;
            pair_free[best] = fin[t];
            owner[t] = best;
            ++count[best];
            if (nb < tn && fin[t] > block_done[si][nb]) block_done[si][nb] = fin[t];
        }
        P.sched_off[0] = 0;
        for (int p = 0; p < pairs; ++p) P.sched_off[p + 1] = (uint16_t)(P.sched_off[p] + count[p]);
        int fill[kChainMaxPairs];
        for (int p = 0; p < pairs; ++p) fill[p] = P.sched_off[p];
        for (int t = 0; t < items; ++t) P.sched[fill[owner[t]]++] = (uint16_t)t;
    }
    if (cache.size() >= 16) cache.erase(cache.begin());
    cache.push_back(Sched{key, std::vector<uint16_t>(P.sched_off, P.sched_off + pairs + 1),
                          std::vector<uint16_t>(P.sched, P.sched + items)});
    cfg.gridDim = dim3(2 * pairs);
    cfg.numAttrs = 2;
    return cudaLaunchKernelEx(&cfg, tc_chain_kernel<OP>, P);
}

cudaError_t launch_tc_chain(const StageArgs *stages, int n, int *done, int *status,
                            unsigned long long *trace, int num_sms, cudaStream_t s)
{
    if (n < 1 || n > kChainMaxStages) return cudaErrorInvalidValue;
    for (int i = 0; i < n; ++i)
        if (stages[i].op != stages[0].op || stages[i].N != stages[0].N || stages[i].M <= 0 ||
            stages[i].K <= 0)
            return cudaErrorInvalidValue;
    switch (stages[0].op) {
    case OP_BF16: return launch_chain_op<OP_BF16>(stages, n, done, status, trace, num_sms, s);
    case OP_I8: return launch_chain_op<OP_I8>(stages, n, done, status, trace, num_sms, s);
    default: return cudaErrorInvalidValue;
    }
}

int chain_max_stages() { return kChainMaxStages; }
int chain_trace_fields() { return kTraceFields; }

}  // namespace fg
