// FP32 (3xTF32) chains whose every stage fits on chip: the panel-resident chain.
//
// The reference runs all stages of a 32-column panel back to back on one core
// and narrows each stage's output straight into the next stage's packed operand
// (multigemm/src/flashgemm.c:123-148; kernel_f32.h:470, f32_save_c_m12n32_2
// writes the next stage's Bc), so intermediates never leave the core. This
// kernel does the same on a B200 SM for chains whose dimensions are all at most
// kPanelKMax (the tall-skinny chains: N up to 65536 columns, 64 x 64 weights):
// a CTA loads a 128-column block of B once (TMA), splits it in place in shared
// memory into the TF32 (hi, lo) pair, and runs every stage on the tensor cores;
// the epilogue of stage i splits its FP32 result into stage i + 1's (hi, lo)
// operand and writes it K-major into shared memory, where stage i + 1's MMAs
// read it. Only the last stage's result goes to global memory. Weights (a few
// KB per stage) stream from L2 through a two-slot TMA ring.
//
// The arithmetic is the grouped 3xTF32 kernel's (fg_group.cu), operation for
// operation: per 32-deep k-block four K = 8 MMAs, each the correction terms
// hi*lo then lo*hi into their own accumulator and hi*hi into the partial sum;
// the partial sum handed to FP32 registers every `kchunk` k-blocks and summed in
// order, the correction added once; the same round-to-nearest TF32 split. The
// results are bit-identical to that kernel's.
//
// Two column blocks are in flight per CTA (two operand buffers), their tiles
// interleaved (block A stage 0, block B stage 0, A 1, B 1, ...), so that one
// block's MMAs run while the other's epilogue drains. Warp 0 is the TMA
// producer, warp 1 allocates TMEM and issues MMAs, warps 2-5 split stage-0
// inputs and run the epilogues. Every wait is bounded (fg_ptx.cuh).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "fg_tc_common.cuh"

namespace fg {

namespace {

constexpr int kPBN = 128;                      // columns per block (MMA N)
constexpr int kPBK = 32;                       // TF32 elements per 128-byte k-block
constexpr int kPKb = kPanelKMax / kPBK;        // k-blocks of the largest operand
constexpr int kPBoxN = 32;                     // MN-major box: 32 columns (128 bytes)
constexpr int kPBoxBytes = kPBoxN * kPBK * 4;  // 4 KB
constexpr int kPKbBytes = kPBN * kPBK * 4;     // one k-block of a (hi or lo) operand: 16 KB
constexpr int kPPartBytes = kPKb * kPKbBytes;  // hi or lo of one block: 32 KB
constexpr int kPSlotBytes = 2 * kPPartBytes;   // (hi, lo) of one block in flight
constexpr int kPWBytes = 128 * 128;            // one k-block of weights (128 rows x 128 B)
constexpr int kPRing = 2;                      // weight ring slots, each (hi, lo)
constexpr int kPXOff = 0;
constexpr int kPWOff = kPXOff + 2 * kPSlotBytes;
constexpr int kPStageOff = kPWOff + kPRing * 2 * kPWBytes;
constexpr int kPBarOff = kPStageOff + kEpiStagingBytes;
constexpr int kPSmem = kPBarOff + 256 + 1024;  // + barriers + alignment slack
constexpr int kPTmemCols = 4 * kPBN;           // 2 partial-sum + 2 correction accumulators
static_assert(kPSmem <= 232448, "shared memory per CTA");
static_assert(kPTmemCols <= 512, "TMEM columns");

// D F32, A TF32, B TF32, A K-major; B MN-major (stage 0, as TMA lands it) or
// K-major (later stages, as the epilogue writes it)
constexpr uint32_t kIdescMN = make_idesc(1, 2, 2, 0, 1, kBM, kPBN);
constexpr uint32_t kIdescK = make_idesc(1, 2, 2, 0, 0, kBM, kPBN);

struct __align__(8) PanelBars {
    uint64_t wfull[kPRing], wempty[kPRing];   // weight ring
    uint64_t xin[2];      // stage-0 input of a block landed in its operand buffer (TMA bytes)
    uint64_t xready[2];   // the operand buffer holds the next tile's B (4 epilogue warps)
    uint64_t xfree[2];    // the MMAs of a block's last stage are done: the buffer may refill
    uint64_t acc_full[2], acc_empty[2];    // partial-sum accumulators
    uint64_t corr_full[2], corr_empty[2];  // correction accumulators
    uint64_t mma_done;
    uint32_t tmem_base;
    int abort;
};
static_assert(sizeof(PanelBars) <= 256, "barrier block");

__device__ __forceinline__ void p_set_abort(PanelBars *b) { *reinterpret_cast<volatile int *>(&b->abort) = 1; }
__device__ __forceinline__ bool p_aborted(PanelBars *b) { return *reinterpret_cast<volatile int *>(&b->abort) != 0; }

// The tiles of one CTA in the order every role walks them: the CTA's blocks
// alternate between operand buffers (slot = position % 2), and the tiles of
// the two slots' current blocks interleave, one tile of each in turn.
struct TileWalk {
    const PanelArgs *g;
    int q0, q1;   // this CTA's blocks: g->blocks[q0 .. q1)
    int pos[2];   // slot s: position (q0 + s, q0 + s + 2, ...) of its current block
    int stage[2];
    int turn;
    __device__ void init(const PanelArgs &args, int cta)
    {
        g = &args;
        q0 = args.off[cta];
        q1 = args.off[cta + 1];
        pos[0] = q0;
        pos[1] = q0 + 1;
        stage[0] = stage[1] = 0;
        turn = 0;
    }
    __device__ int stages_of(int q) const { return g->chains[g->blocks[q] >> 16].n; }
    // Next tile: slot, block position, stage, whether it is the block's last
    // stage, and the next block position of that slot (q1 and beyond: none).
    // false when the CTA has no more tiles.
    __device__ bool next(int &slot, int &q, int &st, bool &last)
    {
        int s = turn;
        if (pos[s] >= q1) s ^= 1;
        if (pos[s] >= q1) return false;
        slot = s;
        q = pos[s];
        st = stage[s];
        last = st + 1 == stages_of(q);
        if (last) {
            pos[s] += 2;
            stage[s] = 0;
        } else {
            ++stage[s];
        }
        turn = s ^ 1;
        return true;
    }
};

// K-major (hi or lo) operand: element (k, n) of a block, 128-byte rows of 32
// k-values per column n, 16-byte chunks swizzled over 8-row atoms (the layout
// a TMA load with 128-byte swizzle gives a K-major operand).
__device__ __forceinline__ uint32_t kmajor_off(int k, int n)
{
    const int kk = k & 31;
    return (uint32_t)((k >> 5) * kPKbBytes + n * 128 + ((((kk >> 2) ^ (n & 7)) << 4)) + (kk & 3) * 4);
}

}  // namespace

__global__ void __launch_bounds__(kThreads, 1) tc_panel_kernel(const __grid_constant__ PanelArgs g)
{
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    PanelBars *bars = reinterpret_cast<PanelBars *>(smem + kPBarOff);
    uint8_t *xbuf = smem + kPXOff;  // slot s: hi at s * kPSlotBytes, lo kPPartBytes later
    uint8_t *wring = smem + kPWOff; // slot r: hi at r * 2 * kPWBytes, lo kPWBytes later
    int *status = g.status;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int r = 0; r < kPRing; ++r) {
            mbar_init(&bars->wfull[r], 1);
            mbar_init(&bars->wempty[r], 1);
        }
        for (int s = 0; s < 2; ++s) {
            mbar_init(&bars->xin[s], 1);
            mbar_init(&bars->xready[s], 4);
            mbar_init(&bars->xfree[s], 1);
            mbar_init(&bars->acc_full[s], 1);
            mbar_init(&bars->acc_empty[s], 4);
            mbar_init(&bars->corr_full[s], 1);
            mbar_init(&bars->corr_empty[s], 4);
        }
        mbar_init(&bars->mma_done, 1);
        bars->abort = 0;
        fence_mbar_init();
    }
    if (warp == 1) tmem_alloc(&bars->tmem_base, kPTmemCols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = bars->tmem_base;

    TileWalk walk;
    walk.init(g, blockIdx.x);

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            int r = 0;
            uint32_t rph = 0;
            uint32_t pending = 0, pending_ph = 0;  // ring slots with loads in flight
            uint32_t xin_pending = 0;              // operand buffers with a load in flight
            uint32_t xin_ph[2] = {0, 0};
            int loaded[2] = {0, 0};                // blocks loaded into each buffer so far
            int slot, q, st;
            bool last;
            while (walk.next(slot, q, st, last)) {
                const uint32_t bq = g.blocks[q];
                const PanelChain &ch = g.chains[bq >> 16];
                const int n0 = (int)(bq & 0xffffu) * kPBN;
                if (st == 0) {
                    // this block's B into the slot's buffer once the slot's previous
                    // block's last MMAs are done
                    if (!mbar_wait(&bars->xfree[slot], (uint32_t)(loaded[slot] & 1) ^ 1u, status,
                                   KERR_WAIT_EMPTY)) {
                        p_set_abort(bars);
                        goto producer_done;
                    }
                    ++loaded[slot];
                    const int nkb = (ch.K[0] + kPBK - 1) / kPBK;
                    int nvb = (ch.N - n0 + kPBoxN - 1) / kPBoxN;  // boxes that start inside N
                    nvb = nvb < kPBN / kPBoxN ? nvb : kPBN / kPBoxN;
                    mbar_arrive_expect_tx(&bars->xin[slot], (uint32_t)(nkb * nvb * kPBoxBytes));
                    uint8_t *x = xbuf + slot * kPSlotBytes;
                    for (int kb = 0; kb < nkb; ++kb)
                        for (int j = 0; j < nvb; ++j)
                            tma_load_2d(x + kb * kPKbBytes + j * kPBoxBytes, &ch.tm_b, &bars->xin[slot],
                                        n0 + j * kPBoxN, kb * kPBK);
                    xin_pending |= 1u << slot;
                    xin_ph[slot] = (uint32_t)((loaded[slot] - 1) & 1);
                }
                const int nkb = (ch.K[st] + kPBK - 1) / kPBK;
                for (int kb = 0; kb < nkb; ++kb) {
                    if (!mbar_wait(&bars->wempty[r], rph ^ 1, status, KERR_WAIT_EMPTY)) {
                        p_set_abort(bars);
                        goto producer_done;
                    }
                    uint8_t *w = wring + r * 2 * kPWBytes;
                    mbar_arrive_expect_tx(&bars->wfull[r], 2u * kPWBytes);
                    tma_load_2d(w, &ch.tm_w[st][0], &bars->wfull[r], kb * kPBK, 0);
                    tma_load_2d(w + kPWBytes, &ch.tm_w[st][1], &bars->wfull[r], kb * kPBK, 0);
                    pending |= 1u << r;
                    pending_ph = (pending_ph & ~(1u << r)) | (rph << r);
                    if (++r == kPRing) {
                        r = 0;
                        rph ^= 1;
                    }
                }
                if (p_aborted(bars)) break;
            }
        producer_done:
            // never leave with copies in flight into this CTA's shared memory
            for (int i = 0; i < kPRing; ++i)
                if (pending & (1u << i))
                    mbar_wait(&bars->wfull[i], (pending_ph >> i) & 1u, status, KERR_WAIT_FULL);
            for (int s = 0; s < 2; ++s)
                if (xin_pending & (1u << s)) mbar_wait(&bars->xin[s], xin_ph[s], status, KERR_WAIT_FULL);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            int r = 0;
            uint32_t rph = 0;
            int acc = 0, cb = 0;
            uint32_t acc_ph = 0, cb_ph = 0;
            int tiles[2] = {0, 0};  // tiles issued per slot: the xready phase to wait for
            int slot, q, st;
            bool last;
            while (walk.next(slot, q, st, last)) {
                const PanelChain &ch = g.chains[g.blocks[q] >> 16];
                if (!mbar_wait(&bars->xready[slot], (uint32_t)(tiles[slot] & 1), status,
                               KERR_WAIT_FULL)) {
                    p_set_abort(bars);
                    goto mma_done;
                }
                ++tiles[slot];
                tc_fence_after();
                const int num_kb = (ch.K[st] + kPBK - 1) / kPBK;
                const int kchunk = ch.kchunk[st] > 0 ? ch.kchunk[st] : num_kb;
                if (!mbar_wait(&bars->corr_empty[cb], cb_ph ^ 1, status, KERR_WAIT_ACC_EMPTY)) {
                    p_set_abort(bars);
                    goto mma_done;
                }
                tc_fence_after();
                const uint32_t c_tmem = tmem_base + 2 * kPBN + cb * kPBN;
                const uint32_t x_hi = smem_u32(xbuf + slot * kPSlotBytes);
                const uint32_t x_lo = x_hi + kPPartBytes;
                for (int kc = 0; kc < num_kb; kc += kchunk) {
                    if (!mbar_wait(&bars->acc_empty[acc], acc_ph ^ 1, status, KERR_WAIT_ACC_EMPTY)) {
                        p_set_abort(bars);
                        goto mma_done;
                    }
                    tc_fence_after();
                    const uint32_t d_tmem = tmem_base + acc * kPBN;
                    const int kend = kc + kchunk < num_kb ? kc + kchunk : num_kb;
                    for (int kb = kc; kb < kend; ++kb) {
                        if (!mbar_wait(&bars->wfull[r], rph, status, KERR_WAIT_FULL)) {
                            p_set_abort(bars);
                            goto mma_done;
                        }
                        tc_fence_after();
                        const uint32_t a_hi = smem_u32(wring + r * 2 * kPWBytes);
                        const uint32_t a_lo = a_hi + kPWBytes;
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const uint64_t ad = smem_desc(a_hi + k * 32, 16, 1024, SMEM_SW128);
                            const uint64_t ad_lo = smem_desc(a_lo + k * 32, 16, 1024, SMEM_SW128);
                            uint64_t bd, bd_lo;
                            uint32_t idesc;
                            if (st == 0) {  // MN-major, 32-byte atoms (as TMA lands B)
                                const uint32_t off = kb * kPKbBytes + k * 8 * 128;
                                bd = smem_desc(x_hi + off, kPBoxBytes, 512, SMEM_SW128_32B);
                                bd_lo = smem_desc(x_lo + off, kPBoxBytes, 512, SMEM_SW128_32B);
                                idesc = kIdescMN;
                            } else {        // K-major (as the epilogue writes it)
                                const uint32_t off = kb * kPKbBytes + k * 32;
                                bd = smem_desc(x_hi + off, 16, 1024, SMEM_SW128);
                                bd_lo = smem_desc(x_lo + off, 16, 1024, SMEM_SW128);
                                idesc = kIdescK;
                            }
                            tc_mma<MmaKind::TF32>(c_tmem, ad, bd_lo, idesc, (kb | k) != 0);
                            tc_mma<MmaKind::TF32>(c_tmem, ad_lo, bd, idesc, 1);
                            tc_mma<MmaKind::TF32>(d_tmem, ad, bd, idesc, (kb != kc || k != 0));
                        }
                        tc_commit(&bars->wempty[r]);
                        if (++r == kPRing) {
                            r = 0;
                            rph ^= 1;
                        }
                    }
                    tc_commit(&bars->acc_full[acc]);
                    if (++acc == 2) {
                        acc = 0;
                        acc_ph ^= 1;
                    }
                }
                tc_commit(&bars->corr_full[cb]);
                if (++cb == 2) {
                    cb = 0;
                    cb_ph ^= 1;
                }
                if (last) tc_commit(&bars->xfree[slot]);  // the buffer may take the next block
                if (p_aborted(bars)) break;
            }
        mma_done:
            tc_commit(&bars->mma_done);
            mbar_wait(&bars->mma_done, 0, status, KERR_WAIT_FULL);
        }
    } else {
        // ------------------------------------------------------------ splits and epilogues
        const int quarter = warp & 3;
        const int et = threadIdx.x - 64;  // 0..127
        const int row = quarter * 32 + lane;  // TMEM lane: output row = next stage's k
        uint8_t *staging = smem + kPStageOff + (warp - 2) * 2 * kStageBufBytes;
        int sbuf = 0;
        int acc = 0, cb = 0;
        uint32_t acc_ph = 0, cb_ph = 0;
        int splits[2] = {0, 0};  // stage-0 inputs split per slot: the xin phase to wait for
        bool ok = true;

        // Split the stage-0 input of the block at position q (in the slot's buffer)
        // into its TF32 (hi, lo) pair in place; then tell the MMA warp.
        auto split = [&](int slot, int q) -> bool {
            if (!mbar_wait(&bars->xin[slot], (uint32_t)(splits[slot] & 1), status, KERR_WAIT_FULL))
                return false;
            ++splits[slot];
            const PanelChain &ch = g.chains[g.blocks[q] >> 16];
            const int bytes = ((ch.K[0] + kPBK - 1) / kPBK) * kPKbBytes;
            uint8_t *hi = xbuf + slot * kPSlotBytes;
            uint8_t *lo = hi + kPPartBytes;
            for (int off = et * 16; off < bytes; off += 128 * 16) {
                const float4 x = *reinterpret_cast<const float4 *>(hi + off);
                float4 h, l;
                h.x = f32_to_tf32_rne(x.x); l.x = f32_to_tf32_rne(x.x - h.x);
                h.y = f32_to_tf32_rne(x.y); l.y = f32_to_tf32_rne(x.y - h.y);
                h.z = f32_to_tf32_rne(x.z); l.z = f32_to_tf32_rne(x.z - h.z);
                h.w = f32_to_tf32_rne(x.w); l.w = f32_to_tf32_rne(x.w - h.w);
                *reinterpret_cast<float4 *>(hi + off) = h;
                *reinterpret_cast<float4 *>(lo + off) = l;
            }
            fence_proxy_async_smem();  // generic writes before the MMAs read them
            __syncwarp();
            if (lane == 0) mbar_arrive(&bars->xready[slot]);
            return true;
        };

        // the first block of each slot
        for (int s = 0; s < 2 && ok; ++s)
            if (walk.q0 + s < walk.q1) ok = split(s, walk.q0 + s);
        int slot, q, st;
        bool last;
        while (ok && walk.next(slot, q, st, last)) {
            const uint32_t bq = g.blocks[q];
            const PanelChain &ch = g.chains[bq >> 16];
            const int n0 = (int)(bq & 0xffffu) * kPBN;
            const int num_kb = (ch.K[st] + kPBK - 1) / kPBK;
            const int kchunk = ch.kchunk[st] > 0 ? ch.kchunk[st] : num_kb;
            float sum[kPBN / 32][32];
#pragma unroll
            for (int c = 0; c < kPBN / 32; ++c)
#pragma unroll
                for (int j = 0; j < 32; ++j) sum[c][j] = 0.f;
            for (int kc = 0; kc < num_kb; kc += kchunk) {
                if (!mbar_wait(&bars->acc_full[acc], acc_ph, status, KERR_WAIT_ACC_FULL)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t t_row = tmem_base + acc * kPBN + ((uint32_t)(quarter * 32) << 16);
#pragma unroll
                for (int c = 0; c < kPBN / 32; ++c) {
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
            if (ok && !mbar_wait(&bars->corr_full[cb], cb_ph, status, KERR_WAIT_ACC_FULL)) ok = false;
            if (!ok) break;
            tc_fence_after();
            {
                const uint32_t t_row =
                    tmem_base + 2 * kPBN + cb * kPBN + ((uint32_t)(quarter * 32) << 16);
#pragma unroll
                for (int c = 0; c < kPBN / 32; ++c) {
                    uint32_t w[32];
                    tmem_ld_32x32b_x32(t_row + c * 32, w);
                    tmem_ld_wait();
#pragma unroll
                    for (int j = 0; j < 32; ++j) sum[c][j] = sum[c][j] + __uint_as_float(w[j]);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bars->corr_empty[cb]);
            if (++cb == 2) {
                cb = 0;
                cb_ph ^= 1;
            }
            const int M = ch.K[st + 1];  // this stage's rows
            if (!last) {
                // the next stage's (hi, lo) operand, K-major, rows k < round_up(M, 32)
                // (rows past M hold the zero products of the zero-filled weight rows)
                if (quarter * 32 < ((M + 31) & ~31)) {
                    uint8_t *hi = xbuf + slot * kPSlotBytes;
                    uint8_t *lo = hi + kPPartBytes;
#pragma unroll
                    for (int c = 0; c < kPBN / 32; ++c)
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const float x = sum[c][j];
                            const float h = f32_to_tf32_rne(x);
                            const uint32_t off = kmajor_off(row, c * 32 + j);
                            *reinterpret_cast<float *>(hi + off) = h;
                            *reinterpret_cast<float *>(lo + off) = f32_to_tf32_rne(x - h);
                        }
                }
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive(&bars->xready[slot]);
            } else {
                // the chain's result: staged TMA stores of 32 columns at a time
                const int warp_row0 = quarter * 32;
                const bool rows_in = warp_row0 < M;
#pragma unroll
                for (int c = 0; c < kPBN / 32; ++c) {
                    const int nc = n0 + c * 32;
                    if (nc >= ch.N) break;  // warp-uniform
                    uint8_t *b0 = staging + sbuf * kStageBufBytes;
                    if (lane == 0) bulk_wait_read<1>();  // this buffer's previous store has read it
                    __syncwarp();
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        st_sw16(b0, lane, 16 * j,
                                make_uint4(__float_as_uint(sum[c][4 * j]), __float_as_uint(sum[c][4 * j + 1]),
                                           __float_as_uint(sum[c][4 * j + 2]),
                                           __float_as_uint(sum[c][4 * j + 3])));
                    sbuf ^= 1;
                    fence_proxy_async_smem();
                    __syncwarp();
                    if (lane == 0 && rows_in) {
                        tma_store_2d(&ch.tm_c, b0, nc, warp_row0);
                        bulk_commit();
                    }
                }
                // this slot's next block, if any: split its stage-0 input
                const int qn = q + 2;
                if (qn < walk.q1 && !split(slot, qn)) ok = false;
            }
            if (p_aborted(bars)) break;
        }
        if (!ok) p_set_abort(bars);
    }

    if (warp >= 2 && lane == 0) bulk_wait<0>();  // staged stores done before shared memory goes
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        tmem_dealloc(tmem_base, kPTmemCols);
    }
}

// ------------------------------------------------------------------ host side

bool panel_eligible(long N, int n, const long *M, const long *K)
{
    if (n < 1 || n > kPanelMaxStages || N <= 0 || N % 4 || N > (long)kPBN * 65535) return false;
    for (int i = 0; i < n; ++i)
        if (M[i] < 1 || M[i] > kPanelKMax || K[i] < 1 || K[i] > kPanelKMax) return false;
    return true;
}

cudaError_t panel_chain_desc(const PanelChainArgs &a, PanelChain &out)
{
    memset(&out, 0, sizeof out);
    if (a.n < 1 || a.n > kPanelMaxStages) return cudaErrorInvalidValue;
    if (!make_map(&out.tm_b, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.B, a.K[0], a.N, a.ldb, kPBoxN,
                  kPBK, CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B))
        return cudaErrorInvalidValue;
    if (!make_map(&out.tm_c, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.C, a.M[a.n - 1], a.N, a.ldc, 32,
                  32))
        return cudaErrorInvalidValue;
    for (int i = 0; i < a.n; ++i) {
        if (!make_map(&out.tm_w[i][0], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.w_hi[i], a.M[i], a.K[i],
                      a.ldw[i], kPBK, kBM) ||
            !make_map(&out.tm_w[i][1], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.w_lo[i], a.M[i], a.K[i],
                      a.ldw[i], kPBK, kBM))
            return cudaErrorInvalidValue;
        out.K[i] = (int)a.K[i];
        out.kchunk[i] = a.kchunk[i];
    }
    out.K[a.n] = (int)a.M[a.n - 1];
    out.n = a.n;
    out.N = (int)a.N;
    return cudaSuccess;
}

int panel_blocks_of(long N) { return (int)((N + kPBN - 1) / kPBN); }

// Blocks to CTAs: longest chains first, each block to the CTA with the least
// work so far (in k-blocks); each CTA's blocks in that order.
void panel_plan(const std::vector<int> &stage_kb, const std::vector<int> &nblocks, int ctas,
                std::vector<uint32_t> &blocks, std::vector<int> &off)
{
    std::vector<std::pair<int, uint32_t>> all;  // (cost, chain << 16 | block)
    for (size_t c = 0; c < nblocks.size(); ++c)
        for (int b = 0; b < nblocks[c]; ++b) all.push_back({stage_kb[c], ((uint32_t)c << 16) | (uint32_t)b});
    std::stable_sort(all.begin(), all.end(), [](auto &x, auto &y) { return x.first > y.first; });
    std::vector<std::vector<uint32_t>> per(ctas);
    std::vector<long> load(ctas, 0);
    for (auto &e : all) {
        int best = 0;
        for (int u = 1; u < ctas; ++u)
            if (load[u] < load[best]) best = u;
        per[best].push_back(e.second);
        load[best] += e.first;
    }
    blocks.clear();
    off.assign(ctas + 1, 0);
    for (int u = 0; u < ctas; ++u) {
        off[u + 1] = off[u] + (int)per[u].size();
        blocks.insert(blocks.end(), per[u].begin(), per[u].end());
    }
}

cudaError_t panel_capacity(int num_sms, int &ctas)
{
    static std::mutex mu;
    static unsigned long long known = 0;
    static int per[64];
    std::lock_guard<std::mutex> lk(mu);
    int dev = 0;
    cudaGetDevice(&dev);
    if (!(known & (1ull << (dev & 63)))) {
        cudaError_t e = cudaFuncSetAttribute(tc_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             kPSmem);
        if (e != cudaSuccess) return e;
        int n = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, tc_panel_kernel, kThreads, kPSmem);
        if (e != cudaSuccess || n < 1) {
            cudaGetLastError();
            return cudaErrorNotSupported;
        }
        per[dev & 63] = n;
        known |= 1ull << (dev & 63);
    }
    ctas = per[dev & 63] * num_sms;
    return cudaSuccess;
}

cudaError_t launch_panel(const PanelChain *chains_dev, const uint32_t *blocks_dev, const int *off_dev,
                         int ctas, int *status, cudaStream_t s)
{
    PanelArgs g;
    g.chains = chains_dev;
    g.blocks = blocks_dev;
    g.off = off_dev;
    g.status = status;
    tc_panel_kernel<<<ctas, kThreads, kPSmem, s>>>(g);
    return cudaGetLastError();
}

}  // namespace fg
