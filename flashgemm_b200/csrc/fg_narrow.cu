// BF16 / INT8 chains with narrow intermediates, kept on chip: the narrow chain.
//
// The reference runs all stages of a 32-column panel back to back on one core
// and narrows each stage's result straight into the next stage's packed
// operand (multigemm/src/flashgemm.c:123-148; kernel_bf16.h:356-391 rounds to
// BF16 into the next Bc, kernel_int8.h:329-385 saturates to int8), so its
// intermediates never leave the core. Its own test chains are of that shape:
// wide activations (N up to 65536), deep first stages (K1 up to 8400) and
// narrow intermediates (M_1, M_2 of 16 to 336; multigemm/test/test_bf16_3.c:14-48).
// This kernel does the same on a B200 SM for chains whose intermediates have at
// most kNarrowRows rows: a CTA owns a 128-column block, streams the first
// stage's weights and activations through a TMA ring, and converts every
// intermediate exactly as the reference does (BF16 round-to-nearest-even or
// int8 saturation, the 2 x 32 / 4 x 32 panel permutation, the INT8 tail rows)
// straight into shared memory, K-major, where the next stage's MMAs read it as
// their B operand. Only the last stage's result is stored.
//
// Tiles are 128 weight rows x 128 columns (cta_group::1); a stage with more
// rows runs several row tiles over the same operand. Two column blocks are in
// flight per CTA (two operand buffers), their stages interleaved so that one
// block's MMAs run while the other's epilogue converts. Warp 0 is the TMA
// producer, warp 1 allocates TMEM and issues MMAs, warps 2-9 run the
// epilogues. Every wait is bounded (fg_ptx.cuh). A CTA owns its column blocks
// entirely, so no CTA waits on another.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "fg_tc_common.cuh"

namespace fg {

namespace {

constexpr int kNBN = 128;               // columns per block (MMA N)
constexpr int kNKbBytes = kNBN * 128;   // one K-major k-block of an operand: 16 KB
constexpr int kNABytes = 128 * 128;     // one weight box: 128 rows x 128 bytes
constexpr int kNAcc = 4;                // TMEM accumulators of 128 columns

template <int OP>
struct NarrowGeo {
    static constexpr int elt = OP == OP_BF16 ? 2 : 1;
    static constexpr int BK = 128 / elt;                   // k per 128-byte k-block
    static constexpr int BOX_N = 128 / elt;                // MN-major box: 128-byte rows
    static constexpr int NBOX = kNBN / BOX_N;              // B boxes per k-block
    static constexpr int BOX_BYTES = BOX_N * BK * elt;     // 8 KB (BF16) / 16 KB (INT8)
    static constexpr int B_BYTES = NBOX * BOX_BYTES;       // 16 KB
    static constexpr int B_KSTEP = (32 / elt) * 128;       // B bytes per MMA k-step (MN-major)
    // D F32 / S32, A BF16 / U8 (K-major), B BF16 / S8: MN-major as TMA lands the
    // first stage's activations, K-major as the epilogue writes an intermediate
    static constexpr uint32_t idesc_mn = OP == OP_BF16 ? make_idesc(1, 1, 1, 0, 1, kBM, kNBN)
                                                       : make_idesc(2, 0, 1, 0, 1, kBM, kNBN);
    static constexpr uint32_t idesc_k = OP == OP_BF16 ? make_idesc(1, 1, 1, 0, 0, kBM, kNBN)
                                                      : make_idesc(2, 0, 1, 0, 0, kBM, kNBN);
    static_assert(kNarrowRows % BK == 0, "intermediates hold whole k-blocks");
};

// Shared memory of a launch (sizes per launch, NarrowArgs): the ring of slots
// (each the weight boxes of one unit's row tiles and, for the first stage, the
// activation boxes they share), the operand buffers (one or two blocks in
// flight), the output staging, the INT8 tail quad, the barriers.
constexpr int kNQuadBytes = 4 * kNBN;
// Epilogue warps per launch: 4 (one per TMEM lane quarter, all 128 columns) or
// 8 (two per quarter, 64 columns each: half the work per warp, but 32 KB more
// staging, so a smaller ring)
__host__ __device__ constexpr int n_threads(int ew) { return 64 + 32 * ew; }
__host__ __device__ constexpr int n_staging(int ew) { return ew * 2 * kStageBufBytes; }
__host__ __device__ constexpr int n_fixed(int ew) { return n_staging(ew) + kNQuadBytes + 256 + 1024; }
constexpr int kNMaxSmem = 232448;

struct __align__(8) NarrowBars {
    uint64_t wfull[kNarrowMaxRing], wempty[kNarrowMaxRing];  // ring
    uint64_t xready[kNarrowMaxX];            // operand buffer holds the next stage's input
    uint64_t acc_full[kNAcc], acc_empty[kNAcc];
    uint64_t epi_sync;                       // the epilogue warps meet (INT8 tails)
    uint64_t mma_done;
    uint32_t tmem_base;
    int abort;
};
static_assert(sizeof(NarrowBars) <= 256, "barrier block");

__device__ __forceinline__ void n_set_abort(NarrowBars *b) { *reinterpret_cast<volatile int *>(&b->abort) = 1; }
__device__ __forceinline__ bool n_aborted(NarrowBars *b) { return *reinterpret_cast<volatile int *>(&b->abort) != 0; }

// The work units of one CTA in the order every role walks them. The CTA owns
// column blocks cta, cta + grid, ...; with X operand buffers (1 to 4) they take
// turns between them (slot = position % X) and the units of the slots' current
// blocks interleave. A unit is a whole intermediate stage (all its row tiles:
// its epilogue overwrites the operand those tiles read, so it waits for all of
// them, and they share each k-block of their B operand) or one row tile of the
// last stage (written to global memory).
struct NarrowWalk {
    const NarrowArgs *g;
    int nblk, xs;
    // per operand buffer s: block position, stage and row tile of its next unit
    // (plain fields, selected by switch: they stay in registers)
    int p0, p1, p2, p3, st0, st1, st2, st3, rw0, rw1, rw2, rw3;
    int turn;
    __device__ void init(const NarrowArgs &args)
    {
        g = &args;
        nblk = (int)blockIdx.x < args.nblocks
                   ? (args.nblocks - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x
                   : 0;
        xs = args.xslots;
        p0 = 0;
        p1 = xs > 1 ? 1 : (1 << 30);
        p2 = xs > 2 ? 2 : (1 << 30);
        p3 = xs > 3 ? 3 : (1 << 30);
        st0 = st1 = st2 = st3 = rw0 = rw1 = rw2 = rw3 = 0;
        turn = 0;
    }
    __device__ int block_of(int j) const { return (int)blockIdx.x + j * (int)gridDim.x; }
    __device__ static int row_tiles(int M) { return (M + 127) / 128; }
    __device__ int pos_of(int s) const { return s == 0 ? p0 : s == 1 ? p1 : s == 2 ? p2 : p3; }
    // Next unit: slot, block position j, stage, first row tile, row tiles; the
    // buffers take turns, a buffer whose blocks are done drops out.
    __device__ bool next(int &slot, int &j, int &st, int &r0, int &nt)
    {
        int s = turn;
        for (int k = 0; k < 4 && pos_of(s) >= nblk; ++k) s = s + 1 < xs ? s + 1 : 0;
        int pos = pos_of(s);
        if (pos >= nblk) return false;
        int stage = s == 0 ? st0 : s == 1 ? st1 : s == 2 ? st2 : st3;
        int row = s == 0 ? rw0 : s == 1 ? rw1 : s == 2 ? rw2 : rw3;
        slot = s;
        j = pos;
        st = stage;
        r0 = row;
        const int R = row_tiles(g->st[st].M);
        bool done_stage;
        if (st + 1 < g->n) {
            nt = R;
            done_stage = true;
        } else {
            nt = 1;
            done_stage = ++row == R;
        }
        if (done_stage) {
            row = 0;
            if (++stage == g->n) {
                stage = 0;
                pos += xs;
            }
        }
        switch (s) {
        case 0: p0 = pos; st0 = stage; rw0 = row; break;
        case 1: p1 = pos; st1 = stage; rw1 = row; break;
        case 2: p2 = pos; st2 = stage; rw2 = row; break;
        default: p3 = pos; st3 = stage; rw3 = row; break;
        }
        turn = s + 1 < xs ? s + 1 : 0;
        return true;
    }
};

// Timeline of a unit (FG_TRACE_DIR): its description, then the roles' stamps.
enum { NT_DESC, NT_PROD_START, NT_PROD_END, NT_MMA_WAIT, NT_MMA_START, NT_MMA_END, NT_EPI_START,
       NT_EPI_END };
__device__ __forceinline__ void ntrace(const NarrowArgs &g, int u, int f, unsigned long long v)
{
    if (g.trace && u < g.trace_units)
        g.trace[((size_t)blockIdx.x * g.trace_units + u) * kNarrowTraceFields + f] = v;
}

// Byte offset of element (k, n) in a K-major operand: 128-byte rows of
// 128 / elt k-values per column n, 16-byte chunks swizzled over 8-row atoms
// (the layout a TMA load with 128-byte swizzle gives a K-major operand).
template <int ELT>
__device__ __forceinline__ uint32_t kmaj(int k, int n)
{
    constexpr int KPB = 128 / ELT;
    const int byte = (k % KPB) * ELT;
    return (uint32_t)((k / KPB) * kNKbBytes + n * 128 + ((((byte >> 4) ^ (n & 7))) << 4) + (byte & 15));
}

// The epilogue warps meet on an mbarrier (bounded wait) rather than a named
// barrier, so that a warp leaving on an error cannot strand the others.
__device__ __forceinline__ bool epi_meet(NarrowBars *bars, uint32_t &ph, int lane, int *status)
{
    __syncwarp();
    if (lane == 0) mbar_arrive(&bars->epi_sync);
    const bool ok = mbar_wait(&bars->epi_sync, ph, status, KERR_WAIT_ACC_FULL);
    ph ^= 1;
    return ok;
}

}  // namespace

template <int OP, int EW>
__global__ void __launch_bounds__(n_threads(EW), 1) tc_narrow_kernel(const __grid_constant__ NarrowArgs g)
{
    constexpr int kNStagingBytes = n_staging(EW);
    constexpr int kNEpiWarps = EW;
    constexpr int CPW = (kNBN / 32) / (EW / 4);  // 32-column chunks per epilogue warp
    using G = NarrowGeo<OP>;
    constexpr MmaKind KIND = OP == OP_BF16 ? MmaKind::F16 : MmaKind::I8;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    uint8_t *ring = smem;                                   // slot r at r * slot_bytes
    uint8_t *xbuf = ring + g.ring * g.slot_bytes;           // operand s at s * x_bytes
    uint8_t *stg0 = xbuf + g.xslots * g.x_bytes;
    uint32_t *quad = reinterpret_cast<uint32_t *>(stg0 + kNStagingBytes);
    NarrowBars *bars = reinterpret_cast<NarrowBars *>(stg0 + kNStagingBytes + kNQuadBytes);
    int *status = g.status;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int RING = g.ring;

    if (threadIdx.x == 0) {
        for (int r = 0; r < RING; ++r) {
            mbar_init(&bars->wfull[r], 1);
            mbar_init(&bars->wempty[r], 1);
        }
        for (int s = 0; s < kNarrowMaxX; ++s) mbar_init(&bars->xready[s], kNEpiWarps);
        for (int a = 0; a < kNAcc; ++a) {
            mbar_init(&bars->acc_full[a], 1);
            mbar_init(&bars->acc_empty[a], kNEpiWarps);
        }
        mbar_init(&bars->epi_sync, kNEpiWarps);
        mbar_init(&bars->mma_done, 1);
        bars->abort = 0;
        fence_mbar_init();
        // the tensor maps into the TMA unit's cache before their first use
        tma_prefetch_desc(&g.tm_b);
        for (int i = 0; i < g.n; ++i) {
            tma_prefetch_desc(&g.st[i].tm_w);
            if (g.st[i].tail_hi > g.st[i].tail_lo) tma_prefetch_desc(&g.st[i].tm_wt);
        }
        tma_prefetch_desc(&g.st[g.n - 1].tm_out);
    }
    if (warp == 1) tmem_alloc(&bars->tmem_base, kNAcc * kNBN);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = bars->tmem_base;

    NarrowWalk walk;
    walk.init(g);

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            int r = 0;
            uint32_t rph = 0;
            uint32_t pending = 0, pending_ph = 0;
            int slot, j, st, r0, nt;
            for (int u = 0; walk.next(slot, j, st, r0, nt); ++u) {
                const NarrowStage &cs = g.st[st];
                const int n0 = walk.block_of(j) * kNBN;
                const int nkb = (cs.K + G::BK - 1) / G::BK;
                if (g.trace) {
                    ntrace(g, u, NT_DESC,
                           (unsigned long long)st | (unsigned long long)j << 8 |
                               (unsigned long long)r0 << 24 | (unsigned long long)nt << 32 |
                               (unsigned long long)smid() << 40);
                    ntrace(g, u, NT_PROD_START, globaltimer_ns());
                }
                int nvb = (g.N - n0 + G::BOX_N - 1) / G::BOX_N;  // boxes that start inside N
                nvb = nvb < G::NBOX ? nvb : G::NBOX;
                for (int kb = 0; kb < nkb; ++kb) {
                    if (!mbar_wait(&bars->wempty[r], rph ^ 1, status, KERR_WAIT_EMPTY)) {
                        n_set_abort(bars);
                        goto producer_done;
                    }
                    uint8_t *slotp = ring + r * g.slot_bytes;
                    const uint32_t tx = nt * kNABytes + (st == 0 ? nvb * G::BOX_BYTES : 0);
                    mbar_arrive_expect_tx(&bars->wfull[r], tx);
                    for (int t = 0; t < nt; ++t) {
                        // the unit's row tile t: weight rows m0 .. m0 + 127
                        const int m0 = (r0 + t) * 128;
                        const bool tail =
                            cs.tail_hi > cs.tail_lo && m0 < cs.tail_hi && m0 + 128 > cs.tail_lo;
                        tma_load_2d(slotp + t * kNABytes, tail ? &cs.tm_wt : &cs.tm_w,
                                    &bars->wfull[r], kb * G::BK, tail ? m0 - cs.tail_row0 : m0);
                    }
                    if (st == 0)  // the first stage's activations, shared by the row tiles
                        for (int jb = 0; jb < nvb; ++jb)
                            tma_load_2d(slotp + g.ra * kNABytes + jb * G::BOX_BYTES, &g.tm_b,
                                        &bars->wfull[r], n0 + jb * G::BOX_N, kb * G::BK);
                    pending |= 1u << r;
                    pending_ph = (pending_ph & ~(1u << r)) | (rph << r);
                    if (++r == RING) {
                        r = 0;
                        rph ^= 1;
                    }
                }
                if (g.trace) ntrace(g, u, NT_PROD_END, globaltimer_ns());
                if (n_aborted(bars)) break;
            }
        producer_done:
            for (int i = 0; i < RING; ++i)
                if (pending & (1u << i))
                    mbar_wait(&bars->wfull[i], (pending_ph >> i) & 1u, status, KERR_WAIT_FULL);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            int r = 0;
            uint32_t rph = 0;
            unsigned tiles = 0;      // tiles issued: accumulator tiles % kNAcc, phase (tiles / kNAcc) & 1
            uint32_t xr = 0;         // bit s: the xready phase to wait for on buffer s
            int slot, j, st, r0, nt;
            for (int u = 0; walk.next(slot, j, st, r0, nt); ++u) {
                const NarrowStage &cs = g.st[st];
                if (g.trace) ntrace(g, u, NT_MMA_WAIT, globaltimer_ns());
                if (st > 0 && r0 == 0) {
                    if (!mbar_wait(&bars->xready[slot], (xr >> slot) & 1u, status,
                                   KERR_WAIT_FULL)) {
                        n_set_abort(bars);
                        goto mma_done;
                    }
                    xr ^= 1u << slot;
                    tc_fence_after();
                }
                for (int t = 0; t < nt; ++t) {  // the unit's accumulators
                    const unsigned tt = tiles + t;
                    if (!mbar_wait(&bars->acc_empty[tt % kNAcc], ((tt / kNAcc) & 1u) ^ 1u, status,
                                   KERR_WAIT_ACC_EMPTY)) {
                        n_set_abort(bars);
                        goto mma_done;
                    }
                }
                tc_fence_after();
                if (g.trace) ntrace(g, u, NT_MMA_START, globaltimer_ns());
                const int nkb = (cs.K + G::BK - 1) / G::BK;
                const uint32_t xb = smem_u32(xbuf + slot * g.x_bytes);
                for (int kb = 0; kb < nkb; ++kb) {
                    if (!mbar_wait(&bars->wfull[r], rph, status, KERR_WAIT_FULL)) {
                        n_set_abort(bars);
                        goto mma_done;
                    }
                    tc_fence_after();
                    const uint32_t s_addr = smem_u32(ring + r * g.slot_bytes);
                    for (int t = 0; t < nt; ++t) {
                        const uint32_t d_tmem = tmem_base + ((tiles + t) % kNAcc) * kNBN;
                        const uint32_t a_addr = s_addr + t * kNABytes;
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const uint64_t ad = smem_desc(a_addr + k * 32, 16, 1024, SMEM_SW128);
                            if (st == 0) {
                                const uint64_t bd =
                                    smem_desc(s_addr + g.ra * kNABytes + k * G::B_KSTEP,
                                              G::BOX_BYTES, 1024, SMEM_SW128);
                                tc_mma<KIND>(d_tmem, ad, bd, G::idesc_mn, (kb | k) != 0);
                            } else {
                                const uint64_t bd =
                                    smem_desc(xb + kb * kNKbBytes + k * 32, 16, 1024, SMEM_SW128);
                                tc_mma<KIND>(d_tmem, ad, bd, G::idesc_k, (kb | k) != 0);
                            }
                        }
                    }
                    tc_commit(&bars->wempty[r]);
                    if (++r == RING) {
                        r = 0;
                        rph ^= 1;
                    }
                }
                for (int t = 0; t < nt; ++t) tc_commit(&bars->acc_full[(tiles + t) % kNAcc]);
                tiles += nt;
                if (g.trace) ntrace(g, u, NT_MMA_END, globaltimer_ns());
                if (n_aborted(bars)) break;
            }
        mma_done:
            tc_commit(&bars->mma_done);
            mbar_wait(&bars->mma_done, 0, status, KERR_WAIT_FULL);
        }
    } else {
        // ------------------------------------------------------------ epilogues (warps 2..9)
        const int quarter = warp & 3;                 // TMEM lanes this warp may read
        const int c_lo = ((warp - 2) >> 2) * CPW;     // its first 32-column chunk
        const bool lead = quarter == 0 && c_lo == 0;  // the warp that stamps the trace
        const int et = threadIdx.x - 64;  // 0..255: below kNBN, this thread's column for the tail quad
        uint8_t *staging = stg0 + (warp - 2) * 2 * kStageBufBytes;
        int sbuf = 0;
        unsigned tiles = 0;
        uint32_t meet_ph = 0;
        bool ok = true;
        int slot, j, st, r0, nt;
        for (int u = 0; ok && walk.next(slot, j, st, r0, nt); ++u) {
            const NarrowStage &cs = g.st[st];
            const bool last = st + 1 == g.n;
            const int n0 = walk.block_of(j) * kNBN;
            uint8_t *xs = xbuf + slot * g.x_bytes;
            const bool tails = OP == OP_I8 && cs.tail_hi > cs.tail_lo;
            // the first stage's input quad comes from global memory: load it
            // before waiting for the accumulators, so the two latencies overlap
            uint32_t qv0 = 0;
            if (tails && st == 0 && et < kNBN && n0 + et < g.N) {
                const uint8_t *b = static_cast<const uint8_t *>(g.b);
                for (int q = 0; q < 4 && q < cs.K; ++q)
                    qv0 |= (uint32_t)b[(size_t)q * g.ldb + n0 + et] << (8 * q);
            }
            // likewise this lane's weight quad 0 of each tail row of the unit
            uint32_t wq_t[2] = {0u, 0u};
            if (tails)
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    const int row = (r0 + t) * 128 + quarter * 32 + lane;
                    if (t < nt && row >= cs.tail_lo && row < cs.tail_hi)
                        wq_t[t] = *reinterpret_cast<const uint32_t *>(
                            cs.w_tail + (size_t)(row - cs.tail_row0) * cs.ld_w_tail + cs.K);
                }
            // every tile of the unit: an intermediate overwrites the operand they read
            for (int t = 0; t < nt && ok; ++t) {
                const unsigned tt = tiles + t;
                ok = mbar_wait(&bars->acc_full[tt % kNAcc], (tt / kNAcc) & 1u, status,
                               KERR_WAIT_ACC_FULL);
            }
            if (!ok) break;
            tc_fence_after();
            if (g.trace && lead && lane == 0) ntrace(g, u, NT_EPI_START, globaltimer_ns());
            // INT8 tail rows add weight quad 0 x input quad 0: the input's first
            // four rows of this block's columns, copied aside first (a later stage's
            // input is the operand buffer this unit overwrites); every warp passes
            // the meeting points alike
            if (tails) {
                if (!(ok = epi_meet(bars, meet_ph, lane, status))) break;
                if (et < kNBN)
                    quad[et] = st > 0 ? *reinterpret_cast<const uint32_t *>(xs + kmaj<1>(0, et)) : qv0;
                if (!(ok = epi_meet(bars, meet_ph, lane, status))) break;
            }
            // rows of the next stage's operand that its MMAs read (k-blocks of BK)
            const int xrows = (cs.M + G::BK - 1) / G::BK * G::BK;
            for (int t = 0; t < nt; ++t) {
                const unsigned tt = tiles + t;
                const int warp_row0 = (r0 + t) * 128 + quarter * 32;
                const int row = warp_row0 + lane;  // stage output row
                const uint32_t t_row =
                    tmem_base + (tt % kNAcc) * kNBN + ((uint32_t)(quarter * 32) << 16);
                const bool tail_row = tails && row >= cs.tail_lo && row < cs.tail_hi;
                const uint32_t wq = t == 0 ? wq_t[0] : wq_t[1];
                // rows written: the result's stored rows; an INT8 intermediate's M
                // rows (the next stage's weights are zero past its K = M, and
                // 0 x anything is 0 in integers); a BF16 intermediate's rows up to
                // the k-block end, zeros past M (a stale NaN x 0 would be NaN)
                bool rows_out = warp_row0 < (last ? cs.out_rows : OP == OP_I8 ? cs.M : xrows);
                if (OP == OP_BF16 && !last && rows_out && warp_row0 >= cs.M) {
                    // a warp wholly past M: its 32 rows of its columns are zero
                    const int kb = warp_row0 / G::BK, c0 = (warp_row0 % G::BK) / 8;
#pragma unroll
                    for (int i = 0; i < 4 * CPW; ++i) {
                        const int idx = lane + 32 * i, n = c_lo * 32 + (idx >> 2), c = c0 + (idx & 3);
                        *reinterpret_cast<uint4 *>(xs + kb * kNKbBytes + n * 128 + ((c ^ (n & 7)) << 4)) =
                            make_uint4(0u, 0u, 0u, 0u);
                    }
                    rows_out = false;
                }
#pragma unroll 1
                for (int c = c_lo; c < c_lo + CPW && rows_out; ++c) {
                    const int lc = c * 32, nc = n0 + lc;
                    if (nc >= g.N) break;  // warp-uniform
                    uint32_t v[32];
                    tmem_ld_32x32b_x32(t_row + c * 32, v);
                    tmem_ld_wait();
                    if (tail_row) {
                        // + sum over q of weight byte q (unsigned) x input byte q
                        // (signed): one mixed-sign dp4a per value, exact in int32
#pragma unroll
                        for (int jj = 0; jj < 32; ++jj) {
                            int r;
                            asm("dp4a.u32.s32 %0, %1, %2, %3;"
                                : "=r"(r)
                                : "r"(wq), "r"(quad[lc + jj]), "r"((int)v[jj]));
                            v[jj] = (uint32_t)r;
                        }
                    }
                    if (last) {
                        // the chain's result: staged TMA store of these 32 columns
                        uint8_t *b0 = staging + sbuf * kStageBufBytes;
                        if (lane == 0) bulk_wait_read<1>();
                        __syncwarp();
#pragma unroll
                        for (int q = 0; q < 8; ++q)
                            st_sw16(b0, lane, 16 * q,
                                    make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]));
                        sbuf ^= 1;
                        fence_proxy_async_smem();
                        __syncwarp();
                        if (lane == 0) {
                            tma_store_2d(&cs.tm_out, b0, nc, warp_row0);
                            bulk_commit();
                        }
                        continue;
                    }
                    // an intermediate: the reference's narrowing and panel permutation,
                    // written K-major into the next stage's operand (k' = output row)
                    const bool full = nc + 32 <= g.N;
                    if constexpr (OP == OP_BF16) {
                        if (cs.permute && full && row < (cs.M & ~1)) {
                            // (2q + h, c) -> (2q + (c & 1), 16h + c / 2)  (kernel_bf16.h:6-32)
                            const int h = row & 1, k0 = row - h;
#pragma unroll
                            for (int u = 0; u < 16; ++u)
                                *reinterpret_cast<uint32_t *>(xs + kmaj<2>(k0, lc + 16 * h + u)) =
                                    pack_bf16x2(v[2 * u], v[2 * u + 1]);
                        } else {
#pragma unroll
                            for (int u = 0; u < 32; ++u)
                                *reinterpret_cast<uint16_t *>(xs + kmaj<2>(row, lc + u)) =
                                    (uint16_t)(pack_bf16x2(v[u], v[u]) & 0xffffu);
                        }
                    } else {
                        if (cs.permute && full && row < (cs.M / 4) * 4) {
                            // (4q + h, c) -> (4q + (c & 3), 8h + c / 4)  (kernel_int8.h:6-50)
                            const int h = row & 3, k0 = row - h;
#pragma unroll
                            for (int u = 0; u < 8; ++u)
                                *reinterpret_cast<uint32_t *>(xs + kmaj<1>(k0, lc + 8 * h + u)) =
                                    pack_s8x4(v[4 * u], v[4 * u + 1], v[4 * u + 2], v[4 * u + 3]);
                        } else if (row < cs.M) {
#pragma unroll
                            for (int u = 0; u < 32; ++u)
                                xs[kmaj<1>(row, lc + u)] = (uint8_t)(pack_s8x4(v[u], 0, 0, 0) & 0xffu);
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&bars->acc_empty[tt % kNAcc]);
            }
            tiles += nt;
            if (g.trace && lead && lane == 0) ntrace(g, u, NT_EPI_END, globaltimer_ns());
            if (!last) {
                // the next stage's input is in place: tell the MMA warp
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive(&bars->xready[slot]);
            }
            if (n_aborted(bars)) break;
        }
        if (!ok) n_set_abort(bars);
    }

    if (warp >= 2 && lane == 0) bulk_wait<0>();
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem_base, kNAcc * kNBN);
    }
}

// ------------------------------------------------------------------ host side

bool narrow_eligible(const StageArgs *st, int n)
{
    if (n < 2 || n > kNarrowMaxStages) return false;
    const int op = st[0].op;
    if (op != OP_BF16 && op != OP_I8) return false;
    const long N = st[0].N;
    if (N < 1 || (N + kNBN - 1) / kNBN > (1l << 30)) return false;
    for (int i = 0; i < n; ++i) {
        if (st[i].op != op || st[i].N != N) return false;
        if (i + 1 < n && (st[i].M > kNarrowRows || st[i].M < 1)) return false;
    }
    return true;
}

// On B200, over the reference's chain table (N 3136..65536, K_1 288..4800):
// INT8 chains run faster narrow at every width (their fused path pays the
// tail-row preparation and an int8 round trip per stage); BF16 chains whose
// 128-column blocks fill fewer than half the SMs run their deep first stage on
// too few SMs and are faster on the fused chain kernel, which splits rows too.
bool narrow_preferred(const StageArgs *st, int n, int num_sms)
{
    (void)n;
    if (st[0].op == OP_I8) return true;
    const long nblk = (st[0].N + kNBN - 1) / kNBN;
    return 2 * nblk >= num_sms;
}

namespace {

// The shared memory layout of a chain: the weight boxes of the widest unit
// (row tiles of the widest intermediate) and the first stage's activations per
// ring slot; operand buffers as deep as the widest intermediate; two column
// blocks in flight when that leaves at least three ring slots, else one.
// Eight epilogue warps where every intermediate is one row tile (measured on
// the reference's chain table: INT8 N = 65536 56 -> 48 us, BF16 44 -> 40 us),
// four where a two-tile unit needs the ring's room (eight there cost a ring slot
// and up to 16 %).
template <int OP>
bool narrow_layout(const StageArgs *st, int n, NarrowArgs &A)
{
    using G = NarrowGeo<OP>;
    int ra = 1, xkb = 1;
    for (int i = 0; i + 1 < n; ++i) {
        ra = std::max(ra, (st[i].M + 127) / 128);
        xkb = std::max(xkb, (st[i].M + G::BK - 1) / G::BK);
    }
    A.ra = ra;
    A.epi_warps = ra == 1 ? 8 : 4;
    A.slot_bytes = ra * kNABytes + G::B_BYTES;
    A.x_bytes = xkb * kNKbBytes;
    const int fixed = n_fixed(A.epi_warps);
    // at most two column blocks in flight (FG_NARROW_XSLOTS=<1..4> overrides):
    // four measured slower on the reference's table (INT8 409 against 389 us,
    // BF16 389 against 383), their smaller ring outweighing the extra overlap
    static const int max_xs = [] {
        const char *v = getenv("FG_NARROW_XSLOTS");
        const int x = v ? atoi(v) : 2;
        return x < 1 ? 1 : x > kNarrowMaxX ? kNarrowMaxX : x;
    }();
    for (int xs = max_xs; xs >= 1; --xs) {
        const int avail = kNMaxSmem - fixed - xs * A.x_bytes;
        const int ring = std::min(kNarrowMaxRing, avail / A.slot_bytes);
        if (ring >= (xs == 2 ? 3 : 2)) {
            A.ring = ring;
            A.xslots = xs;
            A.smem = ring * A.slot_bytes + xs * A.x_bytes + fixed;
            return true;
        }
    }
    return false;
}

template <int OP>
cudaError_t narrow_attr(int smem)
{
    static std::mutex mu;
    static int done[64];
    std::lock_guard<std::mutex> lk(mu);
    int dev = 0;
    cudaGetDevice(&dev);
    if (done[dev & 63] >= smem) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(tc_narrow_kernel<OP, 4>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kNMaxSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(tc_narrow_kernel<OP, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kNMaxSmem);
    if (e != cudaSuccess) return e;
    done[dev & 63] = kNMaxSmem;
    return cudaSuccess;
}

template <int OP>
cudaError_t plan_narrow_op(const StageArgs *st, int n, int num_sms, NarrowArgs &out, int &grid)
{
    using G = NarrowGeo<OP>;
    const CUtensorMapDataType dt = OP == OP_BF16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                                 : CU_TENSOR_MAP_DATA_TYPE_UINT8;
    // parameter blocks of the last few operand sets (tensor maps encoded once)
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    struct Built {
        std::vector<long> key;
        NarrowArgs P;
    };
    static std::vector<Built *> built;
    int dev = 0;
    cudaGetDevice(&dev);
    std::vector<long> key = {dev, num_sms, n};
    for (int i = 0; i < n; ++i) {
        const StageArgs &a = st[i];
        const long v[] = {a.M, a.N, a.K, (long)a.w, a.ld_w, (long)a.x, a.ld_x, a.epi, (long)a.out,
                          a.ld_out, a.permute, a.m_written, a.tail_lo, a.tail_hi,
                          (long)a.w_tail, a.ld_w_tail, a.tail_row0};
        key.insert(key.end(), std::begin(v), std::end(v));
    }
    NarrowArgs *P = nullptr;
    for (size_t i = 0; i < built.size(); ++i)
        if (built[i]->key == key) {
            Built *b = built[i];
            built.erase(built.begin() + i);
            built.push_back(b);
            P = &b->P;
            break;
        }
    if (!P) {
        std::unique_ptr<Built> b(new Built);
        memset(&b->P, 0, sizeof b->P);
        NarrowArgs &A = b->P;
        if (!make_map(&A.tm_b, dt, G::elt, st[0].x, st[0].K, st[0].N, st[0].ld_x, G::BOX_N, G::BK))
            return cudaErrorNotSupported;
        for (int i = 0; i < n; ++i) {
            const StageArgs &a = st[i];
            NarrowStage &cs = A.st[i];
            if (!make_map(&cs.tm_w, dt, G::elt, a.w, a.M, a.K, a.ld_w, G::BK, 128))
                return cudaErrorNotSupported;
            cs.tm_wt = cs.tm_w;
            if (a.tail_hi > a.tail_lo &&
                !make_map(&cs.tm_wt, dt, G::elt, a.w_tail, a.M - a.tail_row0, a.K, a.ld_w_tail,
                          G::BK, 128))
                return cudaErrorNotSupported;
            cs.M = a.M;
            cs.K = a.K;
            cs.permute = a.permute;
            cs.tail_lo = a.tail_lo;
            cs.tail_hi = a.tail_hi;
            cs.tail_row0 = a.tail_row0;
            cs.w_tail = static_cast<const uint8_t *>(a.w_tail);
            cs.ld_w_tail = a.ld_w_tail;
            cs.out_rows = a.m_written;
            if (i + 1 == n && !make_out_map(&cs.tm_out, a)) return cudaErrorNotSupported;
            if (i + 1 < n) cs.tm_out = cs.tm_w;
        }
        if (!narrow_layout<OP>(st, n, A)) return cudaErrorNotSupported;
        A.b = st[0].x;
        A.ldb = st[0].ld_x;
        A.op = OP;
        A.n = n;
        A.N = st[0].N;
        A.nblocks = (st[0].N + kNBN - 1) / kNBN;
        b->key.swap(key);
        if (built.size() >= 8) {
            delete built.front();
            built.erase(built.begin());
        }
        built.push_back(b.release());
        P = &built.back()->P;
    }
    const cudaError_t e = narrow_attr<OP>(P->smem);
    if (e != cudaSuccess) return e;
    out = *P;  // a copy: the cache may drop this entry once the lock is released
    grid = std::min(P->nblocks, num_sms);  // one CTA per SM (shared memory)
    return cudaSuccess;
}

}  // namespace

cudaError_t plan_narrow(const StageArgs *st, int n, int num_sms, NarrowArgs &out, int &grid)
{
    if (!narrow_eligible(st, n)) return cudaErrorNotSupported;
    return st[0].op == OP_BF16 ? plan_narrow_op<OP_BF16>(st, n, num_sms, out, grid)
                               : plan_narrow_op<OP_I8>(st, n, num_sms, out, grid);
}

int narrow_units_per_cta(const NarrowArgs &P, int grid)
{
    const int per_block = P.n - 1 + (P.st[P.n - 1].M + 127) / 128;
    return (P.nblocks + grid - 1) / grid * per_block;
}

cudaError_t launch_narrow(NarrowArgs &P, int grid, int *status, cudaStream_t s)
{
    P.status = status;
    if (P.op == OP_BF16) {
        if (P.epi_warps == 8)
            tc_narrow_kernel<OP_BF16, 8><<<grid, n_threads(8), P.smem, s>>>(P);
        else
            tc_narrow_kernel<OP_BF16, 4><<<grid, n_threads(4), P.smem, s>>>(P);
    } else {
        if (P.epi_warps == 8)
            tc_narrow_kernel<OP_I8, 8><<<grid, n_threads(8), P.smem, s>>>(P);
        else
            tc_narrow_kernel<OP_I8, 4><<<grid, n_threads(4), P.smem, s>>>(P);
    }
    return cudaGetLastError();
}

}  // namespace fg
