// Host-side internals shared by the library's C-ABI files: fg_api.cu (the
// reference entry points, single chains, the weight registry), fg_group_api.cu
// (grouped launches, plans, the autotuner) and fg_serve.cu (the serving loop).
// Not installed; the public interface is in include/.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/flashgemm.h"
#include "../../include/flashgemm_b200.h"
#include "../../include/libshalom.h"
#include "fg_kernels.h"

#define FG_EXPORT extern "C" __attribute__((visibility("default")))

#define CUDA_TRY(expr)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(FG_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_),    \
                        __FILE__, __LINE__);                                             \
    } while (0)

// A registered weight matrix (fg_weights_register).
struct fg_weights_s {
    int dtype;
    int dev;
    long M, K;
    void *main = nullptr;  // A operand layout (BF16 ld % 8, INT8 ld % 16, FP32 ld % 4)
    long ld = 0;
    float *hi = nullptr, *lo = nullptr;  // FP32: 3xTF32 split
    uint8_t *tail = nullptr;             // INT8: reference tail block
    long ld_tail = 0;
    int tail_row0 = 0, tail_lo = 0, tail_hi = 0;
    size_t bytes = 0;
};

namespace fg {
namespace host {

// ---------------------------------------------------------------- status and settings

// Set this thread's status and message (fg_last_status / fg_last_error).
int fail(int st, const char *fmt, ...);
int ok();

extern std::atomic<unsigned long long> g_launches;  // kernels launched (fg_kernel_launches)
extern std::atomic<int> g_prof_on;                  // per-launch profiling on

int semantics();
int f32_algo();
int sgemm_algo();
int tf32_chunk_blocks(long K);

inline long round_up(long x, long a) { return (x + a - 1) / a * a; }
inline bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }

// ---------------------------------------------------------------- host copies

// Pitched host-to-host copies split by rows over a few threads (the caller's
// among them): how pageable operands move to and from pinned staging memory
// fast enough to keep the copy engines and the GPU busy.
class RowCopier {
public:
    explicit RowCopier(int threads);
    ~RowCopier();
    void copy(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width,
              size_t height);

private:
    void run(int part);
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_go_, cv_done_;
    std::atomic<unsigned long long> gen_{0};  // one per posted copy
    std::atomic<int> pending_{0};             // workers still copying the current one
    std::atomic<bool> stop_{false};
    char *dst_ = nullptr;
    const char *src_ = nullptr;
    size_t dpitch_ = 0, spitch_ = 0, width_ = 0, height_ = 0;
    int parts_ = 1;
};

// ---------------------------------------------------------------- per-device context

struct DevCtx {
    int dev = -1;
    int sms = 0;
    cudaStream_t stream = nullptr;  // the library's own stream (host-pointer calls)
    // The stream the library's work currently goes to: the caller's stream for
    // device-pointer calls, the own stream for host-pointer calls. All of the
    // library's earlier work on this device is ordered before its tail (see
    // enter_stream), so waiting for it waits for everything the library issued.
    cudaStream_t work = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    // host-pointer chains: uploads and downloads on their own streams, so that the
    // copies of one column chunk overlap the compute of another
    static constexpr int kCopyChunks = 4;
    cudaStream_t stream_h2d = nullptr, stream_d2h = nullptr;
    cudaEvent_t ev_up[kCopyChunks] = {}, ev_done[kCopyChunks] = {};
    cudaEvent_t ev_down[kCopyChunks] = {};  // a chunk of C reached pinned staging
    // pageable host operands: staged through this pinned buffer (grow-only) by
    // the copier's threads
    char *pin = nullptr;
    size_t pin_cap = 0;
    std::unique_ptr<RowCopier> copier;
    std::mutex mu;
    char *arena = nullptr;
    size_t arena_cap = 0;
    size_t arena_off = 0;
    char *tab = nullptr;     // grouped launches: device copies of their tables
    size_t tab_cap = 0;
    int *status = nullptr;       // device word the kernels report into
    int *status_host = nullptr;  // pinned copy
    // Fused-chain dependency counters: a block zeroed once and carved call after
    // call (every launch gets counters no earlier launch touched), zeroed again in
    // stream order only when it is used up, instead of a memset per call.
    int *ctr = nullptr;
    size_t ctr_cap = 0, ctr_off = 0;
    // per-launch device timing (fg_profile_begin / fg_profile_query)
    struct Rec {
        cudaEvent_t a, b;
        int kind;
        double flops;
    };
    std::vector<Rec> prof;       // records in use
    std::vector<Rec> prof_pool;  // events to reuse
};

int get_ctx(DevCtx **out);
// Scratch arena (grow-only, carved afresh by every call) and the table block of
// grouped launches.
int arena_reserve(DevCtx *c, size_t bytes);
int tab_reserve(DevCtx *c, size_t bytes);
void *arena_take(DevCtx *c, size_t bytes);
inline size_t carve_size(size_t bytes) { return (bytes + 255) & ~(size_t)255; }

// Sequential 256-byte-aligned carving of a caller-owned device block.
struct Carver {
    char *base = nullptr;
    size_t off = 0;
    void *take(size_t bytes)
    {
        off = (off + 255) & ~(size_t)255;
        void *p = base + off;
        off += bytes;
        return p;
    }
};

// ---------------------------------------------------------------- chains

struct Mat {
    const void *p;
    long ld;
};

inline int elt_of(int dtype) { return dtype == FG_DT_INT8 ? 1 : dtype == FG_DT_BF16 ? 2 : 4; }

int check_shapes(int dtype, long N, int n, const long *M, const long *K);
size_t chain_scratch(int dtype, int algo, long N, int n, const long *M, const long *K);
inline double gemm_flops(long M, long N, long K) { return 2.0 * (double)M * (double)N * (double)K; }

// Count a launch; a launch error becomes FG_ERR_CUDA with `what` in the message.
int launch(cudaError_t e, const char *what);

// Launch one kernel through `fn`; while profiling is on, bracket it with CUDA
// events on the stream the kernel runs on.
template <class Fn>
int run_kernel_on(DevCtx *c, cudaStream_t stream, bool capturing, int kind, double flops,
                  const char *what, Fn &&fn)
{
    DevCtx::Rec r{nullptr, nullptr, kind, flops};
    const bool prof = !capturing && g_prof_on.load(std::memory_order_relaxed) != 0;
    if (prof) {
        if (!c->prof_pool.empty()) {
            r.a = c->prof_pool.back().a;
            r.b = c->prof_pool.back().b;
            c->prof_pool.pop_back();
        } else {
            CUDA_TRY(cudaEventCreate(&r.a));
            CUDA_TRY(cudaEventCreate(&r.b));
        }
        CUDA_TRY(cudaEventRecord(r.a, stream));
    }
    const int st = launch(fn(), what);
    if (prof) {
        CUDA_TRY(cudaEventRecord(r.b, stream));
        c->prof.push_back(r);
    }
    return st;
}

template <class Fn>
int run_kernel(DevCtx *c, int kind, double flops, const char *what, Fn &&fn)
{
    DevCtx::Rec r{nullptr, nullptr, kind, flops};
    const bool prof = g_prof_on.load(std::memory_order_relaxed) != 0;
    if (prof) {
        if (!c->prof_pool.empty()) {
            r.a = c->prof_pool.back().a;
            r.b = c->prof_pool.back().b;
            c->prof_pool.pop_back();
        } else {
            CUDA_TRY(cudaEventCreate(&r.a));
            CUDA_TRY(cudaEventCreate(&r.b));
        }
        CUDA_TRY(cudaEventRecord(r.a, c->work));
    }
    const int st = launch(fn(), what);
    if (prof) {
        CUDA_TRY(cudaEventRecord(r.b, c->work));
        c->prof.push_back(r);
    }
    return st;
}

// Weights already laid out for the kernels (the weight registry keeps these):
// w / ld: the A operand (BF16, INT8, or FP32 for the FFMA path); hi / lo:
// the 3xTF32 split (FP32 only); tail: the INT8 reference tail block.
struct PreparedW {
    const void *w;
    long ld;
    const float *hi, *lo;
    long ld_split;
    const uint8_t *tail;
    long ld_tail;
    int tail_row0, tail_lo, tail_hi;
};

// Stage list of a BF16 or INT8 chain: between-stage buffers carved from `cv`
// (null: the context's arena), weight preparations launched on c->stream.
int build_tc_stages(DevCtx *c, int dtype, int sem, void *C, long ldc, Mat b, long N, int n,
                    const Mat *a, const long *M, const long *K, const PreparedW *pw,
                    std::vector<StageArgs> &out, Carver *cv = nullptr);

// Read and clear the device status word (waits for the context's work stream).
int collect_status(DevCtx *c);
// Order the library's stream after `user` on entry, and `user` after it on exit.
int fence_in(DevCtx *c, void *user);
int fence_out(DevCtx *c, void *user);
// Make `s` the work stream: when it differs from the current one, `s` first
// waits (event) for everything issued on the current one. A null `user`
// handle is the legacy default stream.
int enter_stream(DevCtx *c, cudaStream_t s);
inline cudaStream_t user_stream(void *user) { return user ? (cudaStream_t)user : cudaStreamLegacy; }
// `n` zeroed counters for one fused launch on the work stream.
int take_counters(DevCtx *c, size_t n, int **out);

PreparedW prepared_of(const fg_weights_s *w);

// ---------------------------------------------------------------- grouped launches (fg_group_api.cu)

// Everything one grouped launch needs: host tables and their device copies.
struct GroupExec {
    int dtype = 0, algo = 0, kernel = 0, order = 0;
    double flops = 0.0;
    std::vector<GroupLaunch> gls;      // tensor-core launches: one fused, or one per depth
    std::vector<double> gl_flops;
    std::vector<size_t> done_at;       // each launch's counters in `done`
    size_t done_ints = 0;
    int *done = nullptr;
    std::vector<void *> tables;        // device copies of gls[i].tables
    std::vector<SplitJob> splits;      // 3xTF32: activation splits before the group
    SplitJob *splits_dev = nullptr;
    long split_max = 0;
    struct Level {
        std::vector<FfmaJob> jobs;
        FfmaJob *dev = nullptr;
        int tiles = 0, big = 0;
        double flops = 0.0;
    };
    std::vector<Level> levels;         // plain FP32: one grouped launch per depth
    // 3xTF32 chains small enough to run panel-resident (fg_panel.cu): one launch
    std::vector<PanelChain> panel;
    std::vector<uint32_t> panel_blocks;
    std::vector<int> panel_off;
    int panel_ctas = 0;
    double panel_flops = 0.0;
    PanelChain *panel_dev = nullptr;
    uint32_t *panel_blocks_dev = nullptr;
    int *panel_off_dev = nullptr;
    int kernels() const
    {
        return (int)gls.size() + (splits.empty() ? 0 : 1) + (int)levels.size() +
               (panel.empty() ? 0 : 1);
    }
};

// FP32 3xTF32 chains with every dimension at most kPanelKMax run panel-resident
// (FG_PANEL=0: never).
bool panel_enabled();
// Plan the panel launch of gx.panel (blocks to CTAs; at most max_units CTAs, 0: all SMs).
int panel_finish(DevCtx *c, GroupExec &gx, int max_units = 0);

extern std::atomic<int> g_group_kernel, g_group_order;  // fg_set_group_config

size_t group_chain_bytes(int dtype, int algo, long N, int n, const long *M, const long *K);
int group_check(DevCtx *c, int dtype, int nchains, const fg_chain_desc *chains);
size_t group_buf_bytes(int dtype, int algo, int nchains, const fg_chain_desc *chains);
// FG_GROUP_AUTO / FG_ORDER_AUTO resolved: remembered measurement, else the cost model.
void group_resolve(DevCtx *c, int dtype, int algo, int nchains, const fg_chain_desc *chains,
                   int &kernel, int &order);
// Host side of a grouped launch; buffers from `cv`, kernels report into `status`
// (null: the context's word), grids capped at max_units workers (0: all SMs).
int group_build(DevCtx *c, int dtype, int algo, int kernel, int order, int nchains,
                const fg_chain_desc *chains, Carver &cv, GroupExec &gx, int *status = nullptr,
                int max_units = 0);
size_t group_tab_bytes(const GroupExec &gx);
void group_place(GroupExec &gx, Carver &cv);
int group_upload(const GroupExec &gx, cudaStream_t s, bool sync);
int group_launch(DevCtx *c, const GroupExec &gx, cudaStream_t s, bool capturing,
                 int *status = nullptr);

}  // namespace host
}  // namespace fg
