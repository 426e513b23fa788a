// Internal interface between the host shim (fg_api.cpp) and the CUDA kernels.
// Not installed; the public C ABI is in include/.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include <vector>

namespace fg {

// How a tensor-core GEMM stage writes its result.
enum EpiKind : int {
    EPI_F32 = 0,       // final stage, FP32 C (BF16 / TF32 chains, SGEMM)
    EPI_S32 = 1,       // final stage, int32 C (INT8 chain)
    EPI_BF16 = 2,      // between stages: FP32 -> BF16 (RNE), optional panel permutation
    EPI_S8 = 3,        // between stages: int32 -> int8 (saturate), optional panel permutation
    EPI_TF32SPLIT = 4  // between stages: FP32 -> (hi, lo) TF32 pair for the next 3xTF32 stage
};

enum OperandKind : int { OP_BF16 = 0, OP_I8 = 1, OP_TF32X3 = 2 };

// One GEMM stage D[M x N] = W[M x K] * X[K x N]; W row-major with leading
// dimension ld_w, X row-major with leading dimension ld_x (both in elements).
struct StageArgs {
    int op;            // OperandKind
    int M, N, K;
    const void *w;     // weights (TF32X3: hi part)
    const void *w_lo;  // TF32X3: lo part (same ld)
    long ld_w;
    const void *x;     // activations (TF32X3: hi part)
    const void *x_lo;  // TF32X3: lo part (same ld)
    long ld_x;
    int epi;           // EpiKind
    void *out;         // C, or the next stage's activations (TF32SPLIT: hi)
    void *out_lo;      // TF32SPLIT: lo
    long ld_out;
    int permute;       // 1: apply the reference's panel permutation (EPI_BF16 / EPI_S8)
    int m_written;     // rows >= m_written are not stored (INT8 reference semantics)
    int tail_lo;       // INT8 reference tail rows [tail_lo, tail_hi): their weights come from
    int tail_hi;       //   w_tail (rows tail_row0 .. M-1, pre-shifted by one k-quad, first
    const void *w_tail;//   quad kept at [K, K + 4) for the epilogue's correction term)
    long ld_w_tail;
    int tail_row0;
    int kchunk;        // TF32X3: k-blocks (of 32) per FP32 promotion of the partial sum
    int tma_store;     // set by the launchers: the epilogue writes `out` with TMA bulk stores
    int l2_keep;       // 1: `out` is an intermediate stored with an L2 evict-last policy
    int *status;       // device status word (0 = ok)
};

cudaError_t launch_tc_stage(const StageArgs &a, int num_sms, cudaStream_t s);

// A whole BF16 or INT8 chain (stages[0..n) with the same op and N) in one
// persistent launch; `done` holds chain_counter_ints() zeroed ints.
// Returns cudaErrorNotSupported (nothing launched) where the device cannot
// run it; the caller then launches the stages one by one.
// trace (optional, else null): chain_trace_fields() %globaltimer stamps per (item, CTA).
cudaError_t launch_tc_chain(const StageArgs *stages, int n, int *done, int *status,
                            unsigned long long *trace, int num_sms, cudaStream_t s);
int chain_max_stages();
// Time-out self-test (fg_selftest_timeout): two BF16 stages whose second waits
// on counters nothing releases; waits limited to limit_ns for this launch only.
// `done`: 3 * chain_counter_ints(2, ...) zeroed ints.
cudaError_t launch_tc_chain_stuck(const StageArgs *stages, int *done, int *status, int num_sms,
                                  unsigned long long limit_ns, cudaStream_t s);
// Counters a fused chain of these row counts (n stages, N columns) may use.
size_t chain_counter_ints(int n, const long *M, long N);
int chain_trace_fields();

// ------------------------------------------------------------------ grouped launches
//
// Many chains' stages in one persistent launch. Stage i reads the output of
// stage prev[i] (-1: a chain's first stage; prev[i] < i). Every worker (a CTA,
// or a CTA pair) runs its own list of tiles in order; a tile first waits until
// all tiles of the column block it reads are stored (a counter per column block
// of each stage, released by the epilogue warps).

// One tile: stage index and (row block << 16 | column block).
struct WorkEntry {
    uint32_t stage;
    uint32_t mbnb;
};

struct SchedStage {
    int tiles_m, tiles_n;  // tiles of the stage along M and N
    int prev;              // stage it reads (-1: none), earlier in the list
    int done_off;          // its first counter
    double cost;           // estimated duration of one tile (any unit)
    int row_done = 0;      // 1: done per (column block, row tile) at done_off + nb * tiles_m + mb
    int row_major = 0;     // 1: list the stage's tiles row tile by row tile
    double stream = 0.0;   // > 0: input row tile g is needed only `g * stream` after the
                           // tile starts (the previous stage has row_done)
};

// List schedule: stages in dependency depth order, each stage's tiles column
// block by column block (or row tile by row tile); a tile goes to the worker
// that can start it first (the worker is free and the column block it reads is
// estimated done + handoff, or, streaming, each row tile of it is done by the
// time the tile's k-loop reaches it).
// Worker u runs entries[off[u] .. off[u+1]) in that order, so the earliest
// unfinished entry always heads its worker's list and no worker waits forever.
// makespan (optional): the estimated finish time of the last tile.
// starts (optional): each entry's estimated start, in the order of `entries`.
//
// Options (optional argument):
// * feeders: the last `feed_workers` workers take the last `feed_rows` row
//   tiles of every column block of stage `feed_stage` (row tile by row tile,
//   after that stage's other tiles, which they do not take) and no tile of the
//   stage that reads it. The readers, streamed, start on a column block while
//   the feeders still produce its last rows, instead of all waiting for the
//   whole stage.
// * window: the tiles are placed `window` column blocks at a time, every stage
//   of those blocks before the next blocks' (0: each stage whole, in order), so
//   that an intermediate is read back soon after it is written (stages that
//   share the column blocks: one chain).
// The placement order is a topological order of the tiles (a tile's inputs
// come earlier), and every worker runs its tiles in that order, so no worker
// waits forever.
struct SchedOpts {
    int feed_stage = -1;  // -1: no feeders
    int feed_workers = 0;
    int feed_rows = 0;
    int window = 0;
};
void list_schedule(const SchedStage *st, int n, int units, double handoff, std::vector<int> &off,
                   std::vector<WorkEntry> &entries, double *makespan = nullptr,
                   std::vector<double> *starts = nullptr, const SchedOpts *opts = nullptr);

enum GroupKernel : int {
    GK_PAIR = 0,        // BF16 / INT8: CTA pairs, 256 x 256 tiles, 6-stage ring
    GK_SINGLE_256 = 1,  // BF16 / INT8: single CTAs, 128 x 256 tiles, 4-stage ring
    GK_SINGLE_128 = 2,  // BF16 / INT8: single CTAs, 128 x 128 tiles, 6-stage ring;
                        // 3xTF32: 128 x 128 tiles, 3-stage ring (its only kernel)
};

// A planned grouped launch: device tables (copied to device memory as they are,
// at a 256-byte-aligned address) and the launch shape.
struct GroupLaunch {
    int kernel = GK_PAIR;
    int op = 0;
    int ctas = 0;             // CTAs launched (pairs x 2 for GK_PAIR)
    long entries = 0;         // tiles
    size_t done_ints = 0;     // zeroed counters the launch needs
    int dynamic = 0;          // single-CTA kernel: one list taken in turn (counter: last int)
    size_t off_st = 0, off_sched = 0, off_off = 0;  // table offsets in `tables`
    std::vector<unsigned char> tables;
};

// Column width of a kernel's tiles (the unit of its dependency counters).
int group_tile_n(int kernel, int op);
cudaError_t plan_group(const StageArgs *stages, const int *prev, int n, int kernel, int num_sms,
                       GroupLaunch &out);
cudaError_t launch_group(const GroupLaunch &g, const void *tables_dev, int *done, int *status,
                         cudaStream_t s);

// Pair-kernel pieces behind plan_group / launch_group (fg_chain_fused.cu) and
// the single-CTA ones (fg_group.cu).
cudaError_t plan_pair_group(const StageArgs *stages, const int *prev, int n, int num_sms,
                            GroupLaunch &out);
cudaError_t launch_pair_group(const GroupLaunch &g, const void *tables_dev, int *done,
                              int *status, cudaStream_t s);
cudaError_t plan_single_group(const StageArgs *stages, const int *prev, int n, int kernel,
                              int num_sms, GroupLaunch &out);
cudaError_t launch_single_group(const GroupLaunch &g, const void *tables_dev, int *done,
                                int *status, cudaStream_t s);

// ------------------------------------------------------------------ narrow chains
//
// BF16 / INT8 chains whose intermediates have at most kNarrowRows rows keep
// them on chip (fg_narrow.cu): one CTA per 128-column block, the first stage's
// operands streamed through a TMA ring, each intermediate converted as the
// reference does and written K-major into shared memory, only the last
// stage's result stored. Any K_1, any last width.

constexpr int kNarrowRows = 256;
constexpr int kNarrowMaxStages = 8;
constexpr int kNarrowMaxRing = 4;
constexpr int kNarrowMaxX = 4;       // column blocks in flight per CTA, at most

struct alignas(64) NarrowStage {
    CUtensorMap tm_w;    // weights, K-major boxes of 128 rows x 128 bytes
    CUtensorMap tm_wt;   // INT8 reference tail block (else = tm_w)
    CUtensorMap tm_out;  // last stage: the result (staged TMA stores)
    int M, K;
    int permute;         // the reference's panel permutation between stages
    int tail_lo, tail_hi, tail_row0;
    const uint8_t *w_tail;
    long ld_w_tail;
    int out_rows;        // last stage: rows stored (INT8 reference: 4 * floor(M / 4))
};

struct alignas(64) NarrowArgs {
    NarrowStage st[kNarrowMaxStages];
    CUtensorMap tm_b;    // first stage's activations (K_1 x N), MN-major boxes
    const void *b;       // the same, for the INT8 tail correction
    long ldb;
    int n, N, nblocks;
    int op;              // OperandKind
    // shared memory layout of the launch: ring slots of slot_bytes (ra weight
    // boxes, then the first stage's activation boxes), xslots operand buffers
    // of x_bytes (one per column block in flight, 1 to kNarrowMaxX), smem bytes in all
    int ring, slot_bytes, ra, x_bytes, xslots, smem;
    int epi_warps;       // 4 or 8 epilogue warps
    int *status;
    // optional (else null): kNarrowTraceFields %globaltimer stamps per (CTA, unit)
    unsigned long long *trace;
    int trace_units;     // units per CTA the trace holds
};
constexpr int kNarrowTraceFields = 8;

bool narrow_eligible(const StageArgs *st, int n);
// Where the narrow kernel is measured faster than the fused chain kernel.
bool narrow_preferred(const StageArgs *st, int n, int num_sms);
// The launch parameters and grid of a chain's narrow launch (tensor maps kept
// for the last few operand sets); cudaErrorNotSupported when it does not qualify.
cudaError_t plan_narrow(const StageArgs *st, int n, int num_sms, NarrowArgs &out, int &grid);
cudaError_t launch_narrow(NarrowArgs &P, int grid, int *status, cudaStream_t s);
// Work units one CTA of a narrow launch walks at most (the trace's rows per CTA).
int narrow_units_per_cta(const NarrowArgs &P, int grid);

// ------------------------------------------------------------------ panel-resident chains
//
// FP32 (3xTF32) chains whose every dimension (K_1 and every M_i) is at most
// kPanelKMax run with their intermediates in shared memory (fg_panel.cu): one
// CTA per 128-column block, B read once, only the last stage's result written.

constexpr int kPanelKMax = 64;
constexpr int kPanelMaxStages = 8;

// One chain's device descriptor (tensor maps and shapes).
struct alignas(64) PanelChain {
    CUtensorMap tm_b;                        // B: K[0] x N FP32, MN-major boxes
    CUtensorMap tm_w[kPanelMaxStages][2];    // weights (hi, lo), K-major boxes of 64 rows
    float *C;                                // M_last x N FP32, row stride ldc
    long ldc;
    int n;                                   // stages
    int N;
    int K[kPanelMaxStages + 1];              // K[i]: stage i's depth; K[i + 1] = M_i
    int kchunk[kPanelMaxStages];             // k-blocks per FP32 promotion of the partial sum
};

// One launch: every CTA runs blocks[off[cta] .. off[cta + 1]) (chain << 16 | block);
// or, with blocks null, the single chain `one` (carried in the parameters), CTA
// u running its blocks u, u + grid, u + 2 grid, ...
struct PanelArgs {
    const PanelChain *chains;
    const uint32_t *blocks;
    const int *off;
    int *status;
    // optional (else null): kPanelTraceFields %globaltimer stamps per
    // (block position, stage), rows at (position * kPanelMaxStages + stage)
    unsigned long long *trace;
    int one_blocks;      // blocks of `one`
    PanelChain one;
};
constexpr int kPanelTraceFields = 10;

// Host description of one chain for panel_chain_desc (device pointers).
struct PanelChainArgs {
    int n;
    long N;
    const float *B;
    long ldb;
    float *C;
    long ldc;
    const float *w_hi[kPanelMaxStages], *w_lo[kPanelMaxStages];
    long ldw[kPanelMaxStages];
    long M[kPanelMaxStages], K[kPanelMaxStages];
    int kchunk[kPanelMaxStages];
};

bool panel_eligible(long N, int n, const long *M, const long *K);
cudaError_t panel_chain_desc(const PanelChainArgs &a, PanelChain &out);
int panel_blocks_of(long N);
// Blocks of the chains (stage_kb[c]: chain c's k-blocks per block, a cost) to `ctas` CTAs.
void panel_plan(const std::vector<int> &stage_kb, const std::vector<int> &nblocks, int ctas,
                std::vector<uint32_t> &blocks, std::vector<int> &off);
cudaError_t panel_capacity(int num_sms, int &ctas);
cudaError_t launch_panel(const PanelChain *chains_dev, const uint32_t *blocks_dev, const int *off_dev,
                         int ctas, int *status, cudaStream_t s,
                         unsigned long long *trace = nullptr);
// One chain, its description in the launch parameters (no tables): the
// description of the last few operand sets is kept, so repeat calls encode no
// tensor maps.
cudaError_t launch_panel_one(const PanelChainArgs &a, int num_sms, int *status, cudaStream_t s,
                             unsigned long long *trace = nullptr);

// Plain FP32 SGEMM on CUDA cores: C = A * B, one FMA per k in increasing k;
// with kblock > 0 each block of kblock k is summed from zero and added to C.
struct FfmaArgs {
    int M, N, K;
    const float *A; long lda;
    const float *B; long ldb;
    float *C; long ldc;
    int kblock;
};
cudaError_t launch_ffma_sgemm(const FfmaArgs &a, int num_sms, cudaStream_t s);

// FP32 -> (hi, lo) TF32 split of a rows x cols matrix (leading dims ld_in / ld_out).
cudaError_t launch_split_tf32(const float *in, long ld_in, float *hi, float *lo, long ld_out,
                              long rows, long cols, cudaStream_t s);

// INT8 weight preparation: copies W (M x K, ld_in) into dst (ld_out >= K + 4,
// a multiple of 16), shifting rows [tail_lo, tail_hi) left by one k-quad
// (zero-filling the last quad) and keeping their first quad at [K, K + 4).
cudaError_t launch_prep_int8_weights(const int8_t *src, long ld_in, uint8_t *dst, long ld_out,
                                     long M, long K, long tail_lo, long tail_hi,
                                     cudaStream_t s);

// FP32 -> (hi, lo) TF32 splits of many matrices in one launch (jobs in device memory).
struct SplitJob {
    const float *in;
    long ld_in;
    float *hi, *lo;
    long ld_out, rows, cols;
};
cudaError_t launch_split_tf32_jobs(const SplitJob *jobs_dev, int njobs, long max_elems,
                                   cudaStream_t s);

// Plain FP32 SGEMMs of many independent jobs in one launch (jobs in device
// memory; job j owns CTAs [tile0[j], tile0[j + 1]) ).
struct FfmaJob {
    int M, N, K;
    const float *A; long lda;
    const float *B; long ldb;
    float *C; long ldc;
    int tile0;   // first CTA of this job
    int tiles_n; // column tiles of this job
    int vec;     // 16-byte-aligned rows and pointers
};
int ffma_group_tile(int big);  // tile edge of the grouped FFMA kernel (64, or 128 when big)
cudaError_t launch_ffma_group(const FfmaJob *jobs_dev, int njobs, int total_tiles, int big,
                              cudaStream_t s);

// The same preparation for up to 8 matrices in one launch.
struct PrepJob {
    const int8_t *src;
    long ld_in;
    uint8_t *dst;
    long ld_out;
    long M, K, tail_lo, tail_hi;
};
struct PrepJobs {
    PrepJob job[8];
    int n;
};
cudaError_t launch_prep_int8_jobs(const PrepJobs &jobs, cudaStream_t s);

// Fill `count` 32-bit words with `value`.
cudaError_t launch_fill_u32(uint32_t *dst, size_t count, uint32_t value, cudaStream_t s);

}  // namespace fg
