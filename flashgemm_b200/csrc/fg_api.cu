// C ABI of flashgemm-b200: the reference's entry points (flashgemm.h,
// libshalom.h) and the extension API (flashgemm_b200.h), over the CUDA kernels.
//
// Host code only. One context per device holds a stream, a grow-only scratch
// arena and a device status word; a call takes the context's mutex, so calls
// from several host threads are safe and serialised per device (the
// reference's calls share global state and are not reentrant).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/flashgemm.h"
#include "../../include/flashgemm_b200.h"
#include "../../include/libshalom.h"
#include "fg_kernels.h"

#define FG_EXPORT extern "C" __attribute__((visibility("default")))

namespace {

using namespace fg;

// ---------------------------------------------------------------- status

thread_local int t_status = FG_OK;
thread_local char t_msg[512] = "";

int fail(int st, const char *fmt, ...)
{
    t_status = st;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_msg, sizeof t_msg, fmt, ap);
    va_end(ap);
    return st;
}

int ok()
{
    t_status = FG_OK;
    t_msg[0] = 0;
    return FG_OK;
}

#define CUDA_TRY(expr)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(FG_ERR_CUDA, "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_),    \
                        __FILE__, __LINE__);                                             \
    } while (0)

// ---------------------------------------------------------------- settings

int env_choice(const char *name, const char *a, int va, const char *b, int vb, int dflt)
{
    const char *v = getenv(name);
    if (!v) return dflt;
    if (!strcmp(v, a)) return va;
    if (!strcmp(v, b)) return vb;
    return dflt;
}

std::atomic<int> g_sem{-1}, g_f32{-1}, g_sgemm{-1};
std::atomic<unsigned long long> g_launches{0};

int semantics()
{
    int s = g_sem.load();
    if (s < 0) {
        s = env_choice("FG_SEMANTICS", "ref", FG_SEM_REF, "math", FG_SEM_MATH, FG_SEM_REF);
        g_sem.store(s);
    }
    return s;
}
int f32_algo()
{
    int s = g_f32.load();
    if (s < 0) {
        s = env_choice("FG_F32_ALGO", "ffma", FG_F32_FFMA, "3xtf32", FG_F32_3XTF32, FG_F32_3XTF32);
        g_f32.store(s);
    }
    return s;
}
int sgemm_algo()
{
    int s = g_sgemm.load();
    if (s < 0) {
        s = env_choice("FG_SGEMM_ALGO", "ffma", FG_F32_FFMA, "3xtf32", FG_F32_3XTF32, FG_F32_FFMA);
        g_sgemm.store(s);
    }
    return s;
}

inline long round_up(long x, long a) { return (x + a - 1) / a * a; }
inline bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }

// 3xTF32: k-blocks of 32 between FP32 promotions of the tensor-core partial sum.
// The tensor core's FP32 accumulation error grows with the number of MMAs that
// feed one accumulator; promoting every block keeps small-K GEMMs below the
// FFMA loop's own error, and longer chunks do the same for large K, where the
// FFMA error is larger, at a smaller epilogue cost (measured on B200: error
// ratio to FFMA <= 0.9 at K = 48..512 with 1 block, <= 0.5 at K >= 1024 with 3).
// FG_TF32_CHUNK (k elements) overrides the choice.
int tf32_chunk_blocks(long K)
{
    static const long forced = [] {
        const char *v = getenv("FG_TF32_CHUNK");
        return v ? atol(v) : 0l;
    }();
    if (forced > 0) return (int)((forced + 31) / 32);
    return K <= 512 ? 1 : (K <= 2048 ? 2 : 3);
}

// ---------------------------------------------------------------- per-device context

struct DevCtx {
    int dev = -1;
    int sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    std::mutex mu;
    char *arena = nullptr;
    size_t arena_cap = 0;
    size_t arena_off = 0;
    char *tab = nullptr;     // grouped launches: device copies of their tables
    size_t tab_cap = 0;
    int *status = nullptr;       // device word the kernels report into
    int *status_host = nullptr;  // pinned copy
    // per-launch device timing (fg_profile_begin / fg_profile_query)
    struct Rec {
        cudaEvent_t a, b;
        int kind;
        double flops;
    };
    std::vector<Rec> prof;       // records in use
    std::vector<Rec> prof_pool;  // events to reuse
};

std::atomic<int> g_prof_on{0};

std::mutex g_ctx_mu;
DevCtx *g_ctx[64];

int get_ctx(DevCtx **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(FG_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    }
    if (dev < 0 || dev >= 64) return fail(FG_ERR_NO_DEVICE, "device index %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    if (!g_ctx[dev]) {
        cudaDeviceProp prop;
        CUDA_TRY(cudaGetDeviceProperties(&prop, dev));
        if (prop.major != 10)
            return fail(FG_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a",
                        dev, prop.major, prop.minor);
        DevCtx *c = new DevCtx;
        c->dev = dev;
        c->sms = prop.multiProcessorCount;
        CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&c->ev_in, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&c->ev_out, cudaEventDisableTiming));
        CUDA_TRY(cudaMalloc(&c->status, sizeof(int)));
        CUDA_TRY(cudaMemset(c->status, 0, sizeof(int)));
        CUDA_TRY(cudaMallocHost(&c->status_host, sizeof(int)));
        g_ctx[dev] = c;
    }
    *out = g_ctx[dev];
    return FG_OK;
}

// Scratch: ensure capacity (growing only while the stream is idle), then carve.
int arena_reserve(DevCtx *c, size_t bytes)
{
    c->arena_off = 0;
    if (bytes <= c->arena_cap) return FG_OK;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (c->arena) cudaFree(c->arena);
    c->arena = nullptr;
    c->arena_cap = 0;
    size_t cap = bytes + bytes / 4 + (64u << 20);
    cudaError_t e = cudaMalloc(&c->arena, cap);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(FG_ERR_NOMEM, "device scratch of %zu bytes: %s", cap, cudaGetErrorString(e));
    }
    c->arena_cap = cap;
    return FG_OK;
}

// Table block of grouped launches (grow-only, like the arena).
int tab_reserve(DevCtx *c, size_t bytes)
{
    if (bytes <= c->tab_cap) return FG_OK;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (c->tab) cudaFree(c->tab);
    c->tab = nullptr;
    c->tab_cap = 0;
    size_t cap = bytes + bytes / 4 + (1u << 20);
    cudaError_t e = cudaMalloc(&c->tab, cap);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(FG_ERR_NOMEM, "device tables of %zu bytes: %s", cap, cudaGetErrorString(e));
    }
    c->tab_cap = cap;
    return FG_OK;
}

void *arena_take(DevCtx *c, size_t bytes)
{
    size_t off = (c->arena_off + 255) & ~(size_t)255;
    c->arena_off = off + bytes;
    return c->arena + off;
}

size_t carve_size(size_t bytes) { return (bytes + 255) & ~(size_t)255; }

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

// ---------------------------------------------------------------- chain core

struct Mat {
    const void *p;
    long ld;
};

int elt_of(int dtype) { return dtype == FG_DT_INT8 ? 1 : dtype == FG_DT_BF16 ? 2 : 4; }

int check_shapes(int dtype, long N, int n, const long *M, const long *K)
{
    if (n < 1) return fail(FG_ERR_INVALID, "num_gemm must be >= 1 (got %d)", n);
    if (N < 0) return fail(FG_ERR_INVALID, "N must be >= 0");
    for (int i = 0; i < n; ++i) {
        if (M[i] <= 0 || K[i] <= 0)
            return fail(FG_ERR_INVALID, "gemm %d: M and K must be positive", i + 1);
        if (i > 0 && K[i] != M[i - 1])
            return fail(FG_ERR_INVALID, "gemm %d: K (%ld) must equal the previous M (%ld)", i + 1,
                        K[i], M[i - 1]);
        if (M[i] > (1l << 30) || K[i] > (1l << 30) || N > (1l << 30))
            return fail(FG_ERR_INVALID, "gemm %d: dimension too large", i + 1);
    }
    (void)dtype;
    return FG_OK;
}

// Bytes of scratch a chain needs beyond its inputs and output.
size_t chain_scratch(int dtype, int algo, long N, int n, const long *M, const long *K)
{
    const long ldN = round_up(N, 16);
    size_t s = 0;
    long maxM = 0;
    for (int i = 0; i < n - 1; ++i) maxM = M[i] > maxM ? M[i] : maxM;
    if (dtype == FG_DT_INT8 || dtype == FG_DT_BF16) {  // fused-chain completion counters
        s += carve_size((size_t)n * ((N + 255) / 256) * sizeof(int));
        if (getenv("FG_TRACE_DIR")) {  // per-tile timeline of the fused kernel
            size_t items = 0;
            for (int i = 0; i < n; ++i) items += (size_t)((M[i] + 255) / 256) * ((N + 255) / 256);
            s += carve_size(items * 2 * 10 * 8);
        }
    }
    if (dtype == FG_DT_INT8) {
        for (int i = 0; i < n; ++i) {  // padded copy (unaligned rows) + tail block (<= 267 rows)
            s += carve_size((size_t)M[i] * round_up(K[i] + 4, 16));
            s += carve_size((size_t)(M[i] < 272 ? M[i] : 272) * round_up(K[i] + 4, 16));
        }
        s += 2 * carve_size((size_t)maxM * ldN);
    } else if (dtype == FG_DT_BF16) {
        for (int i = 0; i < n; ++i)
            if (K[i] % 8) s += carve_size((size_t)M[i] * round_up(K[i], 8) * 2);
        s += 2 * carve_size((size_t)maxM * ldN * 2);
    } else if (algo == FG_F32_3XTF32) {
        for (int i = 0; i < n; ++i) s += 2 * carve_size((size_t)M[i] * round_up(K[i], 4) * 4);
        s += 2 * carve_size((size_t)K[0] * ldN * 4);                 // split input
        s += 2 * 2 * carve_size((size_t)maxM * ldN * 4);             // ping-pong hi/lo
    } else {
        s += 2 * carve_size((size_t)maxM * ldN * 4);
    }
    return s;
}

int launch(cudaError_t e, const char *what)
{
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (e != cudaSuccess) return fail(FG_ERR_CUDA, "%s launch: %s", what, cudaGetErrorString(e));
    return FG_OK;
}

// Launch one kernel through `fn`; while profiling is on, bracket it with CUDA
// events on the library's stream (the stream the kernel runs on).
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
        CUDA_TRY(cudaEventRecord(r.a, c->stream));
    }
    const int st = launch(fn(), what);
    if (prof) {
        CUDA_TRY(cudaEventRecord(r.b, c->stream));
        c->prof.push_back(r);
    }
    return st;
}

double gemm_flops(long M, long N, long K) { return 2.0 * (double)M * (double)N * (double)K; }

// Whole chain in one fused launch when possible (FG_FUSED=0 turns it off),
// else one tensor-core launch per stage: the per-GEMM path.
std::atomic<int> g_chain_mode{-1};
bool fused_enabled()
{
    int m = g_chain_mode.load();
    if (m < 0) {
        const char *v = getenv("FG_FUSED");
        m = (v && v[0] == '0') ? FG_CHAIN_PER_GEMM : FG_CHAIN_FUSED;
        g_chain_mode.store(m);
    }
    return m == FG_CHAIN_FUSED;
}
bool g_fused_unsupported[64];

int launch_stages(DevCtx *c, int kind, std::vector<StageArgs> &stages, long N)
{
    const int n = (int)stages.size();
    if (fused_enabled() && n <= chain_max_stages() && !g_fused_unsupported[c->dev & 63]) {
        const long tiles_n = (N + 255) / 256;
        int *done = (int *)arena_take(c, (size_t)n * tiles_n * sizeof(int));
        CUDA_TRY(cudaMemsetAsync(done, 0, (size_t)n * tiles_n * sizeof(int), c->stream));
        double fl = 0.0;
        for (auto &st : stages) fl += gemm_flops(st.M, st.N, st.K);
        // FG_TRACE_DIR=<dir>: write a per-tile timeline of every fused launch there
        // (synchronises after the launch: a diagnostic, not for timing runs)
        static const char *trace_dir = getenv("FG_TRACE_DIR");
        unsigned long long *trace = nullptr;
        size_t trace_words = 0;
        if (trace_dir) {
            size_t items = 0;
            for (auto &sa : stages) items += (size_t)((sa.M + 255) / 256) * tiles_n;
            trace_words = items * 2 * chain_trace_fields();
            trace = (unsigned long long *)arena_take(c, trace_words * 8);
            CUDA_TRY(cudaMemsetAsync(trace, 0, trace_words * 8, c->stream));
        }
        cudaError_t le = cudaSuccess;
        int st = run_kernel(c, kind, fl, "fused chain", [&] {
            le = launch_tc_chain(stages.data(), n, done, c->status, trace, c->sms, c->stream);
            return le;
        });
        if (st == FG_OK && trace) {
            std::vector<unsigned long long> h(trace_words);
            CUDA_TRY(cudaMemcpyAsync(h.data(), trace, trace_words * 8, cudaMemcpyDeviceToHost,
                                     c->stream));
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            static int seq = 0;
            char path[1024];
            snprintf(path, sizeof path, "%s/chain_trace_%d.csv", trace_dir, seq++);
            if (FILE *f = fopen(path, "w")) {
                fprintf(f, "q,cta,entry,sm,prod_start,dep_done,prod_end,mma_start,mma_end,"
                           "epi_start,epi_issued,epi_end\n");
                const int nf = chain_trace_fields();
                for (size_t r = 0; r < trace_words / nf; ++r) {
                    fprintf(f, "%zu,%zu", r / 2, r % 2);
                    for (int k = 0; k < nf; ++k) fprintf(f, ",%llu", h[r * nf + k]);
                    fprintf(f, "\n");
                }
                fclose(f);
            }
        }
        if (st == FG_OK) return FG_OK;
        if (le != cudaErrorNotSupported && le != cudaErrorCooperativeLaunchTooLarge &&
            le != cudaErrorInvalidConfiguration)
            return st;
        // this device cannot co-schedule the fused grid: per-stage launches from now on
        cudaGetLastError();
        fprintf(stderr, "flashgemm-b200: fused chain launch unavailable on device %d (%s); "
                        "running one launch per stage\n", c->dev, cudaGetErrorString(le));
        g_launches.fetch_sub(1, std::memory_order_relaxed);
        g_fused_unsupported[c->dev & 63] = true;
        ok();
    }
    for (auto &s : stages) {
        int st = run_kernel(c, kind, gemm_flops(s.M, s.N, s.K),
                            kind == FG_PK_TC_BF16 ? "bf16 stage" : "int8 stage",
                            [&] { return launch_tc_stage(s, c->sms, c->stream); });
        if (st) return st;
    }
    return FG_OK;
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

// Builds the stage list of a BF16 or INT8 chain (between-stage buffers from the
// arena, weight preparations launched on c->stream) without launching the stages.
int build_tc_stages(DevCtx *c, int dtype, int sem, void *C, long ldc, Mat b, long N, int n,
                    const Mat *a, const long *M, const long *K, const PreparedW *pw,
                    std::vector<StageArgs> &out, Carver *cv = nullptr)
{
    auto take = [&](size_t bytes) { return cv ? cv->take(bytes) : arena_take(c, bytes); };
    const long ldN = round_up(N, 16);
    const bool ref = (sem == FG_SEM_REF);
    long maxM = 0;
    for (int i = 0; i < n - 1; ++i) maxM = M[i] > maxM ? M[i] : maxM;
    StageArgs s;
    memset(&s, 0, sizeof s);
    s.status = c->status;
    s.N = (int)N;
    if (dtype == FG_DT_BF16) {
        uint16_t *buf[2] = {nullptr, nullptr};
        if (n > 1) {
            buf[0] = (uint16_t *)take((size_t)maxM * ldN * 2);
            buf[1] = (uint16_t *)take((size_t)maxM * ldN * 2);
        }
        const void *x = b.p;
        long ldx = b.ld;
        std::vector<StageArgs> stages;
        for (int i = 0; i < n; ++i) {
            const void *w = pw ? pw[i].w : a[i].p;
            long ldw = pw ? pw[i].ld : a[i].ld;
            if ((ldw % 8) || ((uintptr_t)w % 16)) {
                const long ldk = round_up(K[i], 8);
                void *wp = take((size_t)M[i] * ldk * 2);
                CUDA_TRY(cudaMemsetAsync(wp, 0, (size_t)M[i] * ldk * 2, c->stream));
                CUDA_TRY(cudaMemcpy2DAsync(wp, ldk * 2, w, ldw * 2, K[i] * 2, M[i],
                                           cudaMemcpyDeviceToDevice, c->stream));
                w = wp;
                ldw = ldk;
            }
            const bool last = (i == n - 1);
            s.op = OP_BF16;
            s.M = (int)M[i]; s.K = (int)K[i];
            s.w = w; s.ld_w = ldw;
            s.x = x; s.ld_x = ldx;
            s.epi = last ? EPI_F32 : EPI_BF16;
            s.out = last ? C : (void *)buf[i & 1];
            s.ld_out = last ? ldc : ldN;
            s.permute = ref ? 1 : 0;
            s.m_written = (int)M[i];
            s.tail_lo = s.tail_hi = 0;
            stages.push_back(s);
            x = s.out;
            ldx = s.ld_out;
        }
        out = std::move(stages);
        return FG_OK;
    }

    // INT8
    {
        uint8_t *buf[2] = {nullptr, nullptr};
        if (n > 1) {
            buf[0] = (uint8_t *)take((size_t)maxM * ldN);
            buf[1] = (uint8_t *)take((size_t)maxM * ldN);
        }
        const void *x = b.p;
        long ldx = b.ld;
        std::vector<StageArgs> stages;
        PrepJobs jobs;
        jobs.n = 0;
        for (int i = 0; i < n; ++i) {
            const long Mi = M[i], Ki = K[i];
            // reference tail rows (multigemm/src/kernel_int8.h:771-1057): only with
            // whole k-quads; other K leave the reference undefined and get no shift
            long tail_lo = 0, tail_hi = 0;
            if (ref && Ki % 4 == 0 && Ki >= 4) {
                tail_lo = (Mi / 12) * 12;
                tail_hi = (Mi / 4) * 4;
            }
            // Weights go to the MMA as they are when their rows are 16-byte aligned
            // (TMA); otherwise through a padded copy. Tail rows always come from a
            // prepared copy of the 256-row block that holds them.
            const long ldw = round_up(Ki + 4, 16);
            const void *wmain = pw ? pw[i].w : a[i].p;
            long ldmain = pw ? pw[i].ld : a[i].ld;
            if ((ldmain % 16) || !aligned16(wmain)) {
                uint8_t *wp = (uint8_t *)take((size_t)Mi * ldw);
                int st = run_kernel(c, FG_PK_AUX, 0.0, "int8 weight copy", [&] {
                    return launch_prep_int8_weights((const int8_t *)a[i].p, a[i].ld, wp, ldw, Mi,
                                                    Ki, 0, 0, c->stream);
                });
                if (st) return st;
                wmain = wp;
                ldmain = ldw;
            }
            s.w_tail = nullptr;
            s.ld_w_tail = 0;
            s.tail_row0 = 0;
            if (tail_hi > tail_lo && pw && pw[i].tail) {  // prepared at registration
                s.w_tail = pw[i].tail;
                s.ld_w_tail = pw[i].ld_tail;
                s.tail_row0 = pw[i].tail_row0;
            } else if (tail_hi > tail_lo) {
                const long row0 = (tail_lo / 256) * 256;
                uint8_t *wt = (uint8_t *)take((size_t)(Mi - row0) * ldw);
                if (jobs.n == 8) {  // flush a full batch
                    int st = run_kernel(c, FG_PK_AUX, 0.0, "int8 tail-row prep",
                                        [&] { return launch_prep_int8_jobs(jobs, c->stream); });
                    if (st) return st;
                    jobs.n = 0;
                }
                jobs.job[jobs.n++] = PrepJob{(const int8_t *)a[i].p + row0 * a[i].ld, a[i].ld, wt, ldw,
                                             Mi - row0, Ki, tail_lo - row0, tail_hi - row0};
                s.w_tail = wt;
                s.ld_w_tail = ldw;
                s.tail_row0 = (int)row0;
            }
            const bool last = (i == n - 1);
            s.op = OP_I8;
            s.M = (int)Mi; s.K = (int)Ki;
            s.w = wmain; s.ld_w = ldmain;
            s.x = x; s.ld_x = ldx;
            s.epi = last ? EPI_S32 : EPI_S8;
            s.out = last ? C : (void *)buf[i & 1];
            s.ld_out = last ? ldc : ldN;
            s.permute = ref ? 1 : 0;
            s.m_written = (last && ref) ? (int)((Mi / 4) * 4) : (int)Mi;
            s.tail_lo = (int)tail_lo;
            s.tail_hi = (int)tail_hi;
            stages.push_back(s);
            x = s.out;
            ldx = s.ld_out;
        }
        if (jobs.n) {  // all tail blocks of the chain in one launch
            int st = run_kernel(c, FG_PK_AUX, 0.0, "int8 tail-row prep",
                                [&] { return launch_prep_int8_jobs(jobs, c->stream); });
            if (st) return st;
        }
        out = std::move(stages);
        return FG_OK;
    }
    return fail(FG_ERR_INVALID, "not a tensor-core chain dtype");
}

// Runs the chain on c->stream. Device operands: B (K[0] x N, ld b.ld),
// A[i] (M[i] x K[i], ld a[i].ld, 16-byte-aligned rows where the tensor path
// needs them), C (M[n-1] x N, ld ldc). Scratch must already be reserved.
int run_chain(DevCtx *c, int dtype, int sem, int algo, void *C, long ldc, Mat b, long N, int n,
              const Mat *a, const long *M, const long *K, const PreparedW *pw = nullptr)
{
    const long ldN = round_up(N, 16);
    long maxM = 0;
    for (int i = 0; i < n - 1; ++i) maxM = M[i] > maxM ? M[i] : maxM;

    if (dtype == FG_DT_F32 && algo == FG_F32_FFMA) {
        float *buf[2] = {nullptr, nullptr};
        if (n > 1) {
            buf[0] = (float *)arena_take(c, (size_t)maxM * ldN * 4);
            buf[1] = (float *)arena_take(c, (size_t)maxM * ldN * 4);
        }
        const float *x = (const float *)b.p;
        long ldx = b.ld;
        for (int i = 0; i < n; ++i) {
            FfmaArgs f;
            f.M = (int)M[i]; f.N = (int)N; f.K = (int)K[i];
            f.A = pw ? (const float *)pw[i].w : (const float *)a[i].p;
            f.lda = pw ? pw[i].ld : a[i].ld;
            f.B = x; f.ldb = ldx;
            const bool last = (i == n - 1);
            f.C = last ? (float *)C : buf[i & 1];
            f.ldc = last ? ldc : ldN;
            f.kblock = 0;  // the multigemm FP32 chain does not split K (kernel_f32.h:3)
            int st = run_kernel(c, FG_PK_FFMA, gemm_flops(M[i], N, K[i]), "ffma stage",
                                [&] { return launch_ffma_sgemm(f, c->sms, c->stream); });
            if (st) return st;
            x = f.C;
            ldx = f.ldc;
        }
        return FG_OK;
    }

    StageArgs s;
    memset(&s, 0, sizeof s);
    s.status = c->status;
    s.N = (int)N;

    if (dtype == FG_DT_F32) {  // 3xTF32
        std::vector<const float *> wh(n), wl(n);
        std::vector<long> wld(n);
        for (int i = 0; i < n; ++i) {
            const long ldk = round_up(K[i], 4);
            wld[i] = ldk;
            if (pw) {
                wh[i] = pw[i].hi;
                wl[i] = pw[i].lo;
                wld[i] = pw[i].ld_split;
                continue;
            }
            float *h = (float *)arena_take(c, (size_t)M[i] * ldk * 4);
            float *l = (float *)arena_take(c, (size_t)M[i] * ldk * 4);
            wh[i] = h;
            wl[i] = l;
            int st = run_kernel(c, FG_PK_AUX, 0.0, "tf32 split (weights)", [&] {
                return launch_split_tf32((const float *)a[i].p, a[i].ld, h, l, ldk, M[i], K[i],
                                         c->stream);
            });
            if (st) return st;
        }
        float *xh = (float *)arena_take(c, (size_t)K[0] * ldN * 4);
        float *xl = (float *)arena_take(c, (size_t)K[0] * ldN * 4);
        int st = run_kernel(c, FG_PK_AUX, 0.0, "tf32 split (activations)", [&] {
            return launch_split_tf32((const float *)b.p, b.ld, xh, xl, ldN, K[0], N, c->stream);
        });
        if (st) return st;
        float *ph[2] = {nullptr, nullptr}, *pl[2] = {nullptr, nullptr};
        if (n > 1)
            for (int j = 0; j < 2; ++j) {
                ph[j] = (float *)arena_take(c, (size_t)maxM * ldN * 4);
                pl[j] = (float *)arena_take(c, (size_t)maxM * ldN * 4);
            }
        for (int i = 0; i < n; ++i) {
            const bool last = (i == n - 1);
            s.op = OP_TF32X3;
            s.M = (int)M[i]; s.K = (int)K[i];
            s.w = wh[i]; s.w_lo = wl[i]; s.ld_w = wld[i];
            s.x = xh; s.x_lo = xl; s.ld_x = ldN;
            s.epi = last ? EPI_F32 : EPI_TF32SPLIT;
            s.out = last ? C : (void *)ph[i & 1];
            s.out_lo = last ? nullptr : (void *)pl[i & 1];
            s.ld_out = last ? ldc : ldN;
            s.m_written = (int)M[i];
            s.tail_lo = s.tail_hi = 0;
            s.kchunk = tf32_chunk_blocks(K[i]);
            st = run_kernel(c, FG_PK_TC_TF32X3, gemm_flops(M[i], N, K[i]), "tf32x3 stage",
                            [&] { return launch_tc_stage(s, c->sms, c->stream); });
            if (st) return st;
            xh = ph[i & 1];
            xl = pl[i & 1];
        }
        return FG_OK;
    }

    {
        std::vector<StageArgs> stages;
        int st = build_tc_stages(c, dtype, sem, C, ldc, b, N, n, a, M, K, pw, stages);
        if (st) return st;
        return launch_stages(c, dtype == FG_DT_BF16 ? FG_PK_TC_BF16 : FG_PK_TC_I8, stages, N);
    }
}

// Read and clear the device status word (the stream must be idle).
int collect_status(DevCtx *c)
{
    CUDA_TRY(cudaMemcpyAsync(c->status_host, c->status, sizeof(int), cudaMemcpyDeviceToHost,
                             c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    const int code = *c->status_host;
    if (code) {
        CUDA_TRY(cudaMemsetAsync(c->status, 0, sizeof(int), c->stream));
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        return fail(FG_ERR_TIMEOUT, "a kernel's pipeline wait ran out (code 0x%x)", code);
    }
    return FG_OK;
}

// Host-pointer chain: stage operands into device scratch, run, copy C back.
int host_chain(int dtype, void *C, const void *B, long N, int n, const void *const *A,
               const long *M, const long *K)
{
    int st = check_shapes(dtype, N, n, M, K);
    if (st) return st;
    for (int i = 0; i < n; ++i)
        if (K[i] % 2 != 0) {
            // same message and behaviour as the reference (flashgemm.c:13-22, :64-68)
            printf("K must be a multiple of 2\n");
            printf("Dimension error for gemm %d\n", i + 1);
            return fail(FG_ERR_INVALID, "gemm %d: K must be a multiple of 2", i + 1);
        }
    if (N == 0) return ok();
    DevCtx *c;
    if ((st = get_ctx(&c))) return st;
    std::lock_guard<std::mutex> lk(c->mu);
    const int elt = elt_of(dtype);
    const int sem = semantics();
    const int algo = f32_algo();
    const long ldN = round_up(N, 16);
    const int out_elt = 4;
    size_t need = carve_size((size_t)K[0] * ldN * elt) + carve_size((size_t)M[n - 1] * ldN * out_elt);
    std::vector<long> lda(n);
    for (int i = 0; i < n; ++i) {
        lda[i] = round_up(K[i], 16 / elt);
        need += carve_size((size_t)M[i] * lda[i] * elt);
    }
    need += chain_scratch(dtype, algo, N, n, M, K) + 4096;
    if ((st = arena_reserve(c, need))) return st;

    void *bd = arena_take(c, (size_t)K[0] * ldN * elt);
    CUDA_TRY(cudaMemcpy2DAsync(bd, ldN * elt, B, N * elt, N * elt, K[0], cudaMemcpyHostToDevice,
                               c->stream));
    std::vector<Mat> ad(n);
    for (int i = 0; i < n; ++i) {
        void *p = arena_take(c, (size_t)M[i] * lda[i] * elt);
        CUDA_TRY(cudaMemcpy2DAsync(p, lda[i] * elt, A[i], K[i] * elt, K[i] * elt, M[i],
                                   cudaMemcpyHostToDevice, c->stream));
        ad[i] = Mat{p, lda[i]};
    }
    void *cd = arena_take(c, (size_t)M[n - 1] * ldN * out_elt);
    if ((st = run_chain(c, dtype, sem, algo, cd, ldN, Mat{bd, ldN}, N, n, ad.data(), M, K)))
        return st;
    // INT8 reference semantics leave rows >= 4 * floor(M / 4) of C untouched
    // (multigemm/src/kernel_int8.h:943-945)
    long rows = M[n - 1];
    if (dtype == FG_DT_INT8 && sem == FG_SEM_REF) rows = (rows / 4) * 4;
    if (rows > 0)
        CUDA_TRY(cudaMemcpy2DAsync(C, N * out_elt, cd, ldN * out_elt, N * out_elt, rows,
                                   cudaMemcpyDeviceToHost, c->stream));
    if ((st = collect_status(c))) return st;
    return ok();
}

int chain_va(int dtype, void *C, const void *B, long N, int num_gemm, va_list ap)
{
    if (num_gemm < 1 || num_gemm > 4096)
        return fail(FG_ERR_INVALID, "num_gemm must be in [1, 4096] (got %d)", num_gemm);
    std::vector<const void *> A(num_gemm);
    std::vector<long> M(num_gemm), K(num_gemm);
    for (int i = 0; i < num_gemm; ++i) {  // flashgemm.c:54-61: (T *A_i, long M_i, long K_i)
        A[i] = va_arg(ap, const void *);
        M[i] = va_arg(ap, long);
        K[i] = va_arg(ap, long);
    }
    return host_chain(dtype, C, B, N, num_gemm, A.data(), M.data(), K.data());
}

// ---------------------------------------------------------------- SGEMM

int run_sgemm(DevCtx *c, int algo, float *C, long ldc, const float *A, long lda, const float *B,
              long ldb, long M, long N, long K, int kblock)
{
    if (algo == FG_F32_FFMA) {
        FfmaArgs f;
        f.M = (int)M; f.N = (int)N; f.K = (int)K;
        f.A = A; f.lda = lda; f.B = B; f.ldb = ldb; f.C = C; f.ldc = ldc;
        f.kblock = kblock;
        return run_kernel(c, FG_PK_FFMA, gemm_flops(M, N, K), "ffma sgemm",
                          [&] { return launch_ffma_sgemm(f, c->sms, c->stream); });
    }
    Mat a{A, lda};
    return run_chain(c, FG_DT_F32, FG_SEM_MATH, FG_F32_3XTF32, C, ldc, Mat{B, ldb}, N, 1, &a, &M, &K);
}

int host_sgemm(float *C, const float *A, const float *B, long M, long N, long K)
{
    if (M < 0 || N < 0 || K < 0) return fail(FG_ERR_INVALID, "negative dimension");
    if (M == 0 || N == 0) return ok();
    if (M > (1l << 30) || N > (1l << 30) || K > (1l << 30))
        return fail(FG_ERR_INVALID, "dimension too large");
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    std::lock_guard<std::mutex> lk(c->mu);
    const int algo = K == 0 ? FG_F32_FFMA : sgemm_algo();
    const long ldk = round_up(K > 0 ? K : 1, 4), ldn = round_up(N, 4);
    size_t need = carve_size((size_t)M * ldk * 4) + carve_size((size_t)K * ldn * 4) +
                  carve_size((size_t)M * ldn * 4) + 4096;
    if (algo == FG_F32_3XTF32) {
        long Ms[1] = {M}, Ks[1] = {K};
        need += chain_scratch(FG_DT_F32, algo, N, 1, Ms, Ks);
    }
    if ((st = arena_reserve(c, need))) return st;
    float *ad = (float *)arena_take(c, (size_t)M * ldk * 4);
    float *bd = (float *)arena_take(c, (size_t)(K > 0 ? K : 1) * ldn * 4);
    float *cd = (float *)arena_take(c, (size_t)M * ldn * 4);
    if (K > 0) {
        CUDA_TRY(cudaMemcpy2DAsync(ad, ldk * 4, A, K * 4, K * 4, M, cudaMemcpyHostToDevice, c->stream));
        CUDA_TRY(cudaMemcpy2DAsync(bd, ldn * 4, B, N * 4, N * 4, K, cudaMemcpyHostToDevice, c->stream));
    }
    // singlegemm blocks K by GEMM_K = 2048 and adds the partial sums into C
    // (singlegemm/src/NN_mp.h:13, :247)
    if ((st = run_sgemm(c, algo, cd, ldn, ad, ldk, bd, ldn, M, N, K, 2048))) return st;
    CUDA_TRY(cudaMemcpy2DAsync(C, N * 4, cd, ldn * 4, N * 4, M, cudaMemcpyDeviceToHost, c->stream));
    if ((st = collect_status(c))) return st;
    return ok();
}

int g_shalom_threads = 24;

// Order the library's stream after `user` on entry, and `user` after it on exit.
// A null handle is CUDA's legacy default stream (the library's own stream is
// non-blocking, so it is not ordered with the default stream implicitly).
int fence_in(DevCtx *c, void *user)
{
    if (!user) user = (void *)cudaStreamLegacy;
    CUDA_TRY(cudaEventRecord(c->ev_in, (cudaStream_t)user));
    CUDA_TRY(cudaStreamWaitEvent(c->stream, c->ev_in, 0));
    return FG_OK;
}
int fence_out(DevCtx *c, void *user)
{
    if (!user) user = (void *)cudaStreamLegacy;
    CUDA_TRY(cudaEventRecord(c->ev_out, c->stream));
    CUDA_TRY(cudaStreamWaitEvent((cudaStream_t)user, c->ev_out, 0));
    return FG_OK;
}

}  // namespace

// ---------------------------------------------------------------- weight registry

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

namespace {

void free_weights(fg_weights_s *w)
{
    if (!w) return;
    cudaFree(w->main);
    cudaFree(w->hi);
    cudaFree(w->lo);
    cudaFree(w->tail);
    delete w;
}

int register_weights(int dtype, const void *A, long M, long K, int where, fg_weights_s **out)
{
    if (dtype != FG_DT_F32 && dtype != FG_DT_BF16 && dtype != FG_DT_INT8)
        return fail(FG_ERR_INVALID, "unknown dtype %d", dtype);
    if (!A || !out) return fail(FG_ERR_INVALID, "null pointer");
    if (M <= 0 || K <= 0 || M > (1l << 30) || K > (1l << 30))
        return fail(FG_ERR_INVALID, "M and K must be positive");
    if (where != FG_MEM_HOST && where != FG_MEM_DEVICE)
        return fail(FG_ERR_INVALID, "where must be FG_MEM_HOST or FG_MEM_DEVICE");
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    std::lock_guard<std::mutex> lk(c->mu);
    const int elt = elt_of(dtype);
    fg_weights_s *w = new fg_weights_s;
    w->dtype = dtype;
    w->dev = c->dev;
    w->M = M;
    w->K = K;
    w->ld = round_up(K, 16 / elt);
    auto alloc = [&](void **p, size_t bytes) -> int {
        cudaError_t e = cudaMalloc(p, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(FG_ERR_NOMEM, "weights: %zu bytes: %s", bytes, cudaGetErrorString(e));
        }
        w->bytes += bytes;
        return FG_OK;
    };
    const size_t main_bytes = (size_t)M * w->ld * elt;
    if (where == FG_MEM_DEVICE) {
        // the source may still be written by work on any stream: registration is
        // a one-time step, so it waits for the device to be idle
        cudaError_t e0 = cudaDeviceSynchronize();
        if (e0 != cudaSuccess) {
            delete w;
            return fail(FG_ERR_CUDA, "weights: %s", cudaGetErrorString(e0));
        }
    }
    if ((st = alloc(&w->main, main_bytes))) {
        free_weights(w);
        return st;
    }
    cudaError_t e = cudaMemsetAsync(w->main, 0, main_bytes, c->stream);
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(w->main, w->ld * elt, A, K * elt, K * elt, M,
                              where == FG_MEM_HOST ? cudaMemcpyHostToDevice
                                                   : cudaMemcpyDeviceToDevice,
                              c->stream);
    if (e != cudaSuccess) {
        free_weights(w);
        return fail(FG_ERR_CUDA, "weights copy: %s", cudaGetErrorString(e));
    }
    if (dtype == FG_DT_F32) {
        const size_t b = (size_t)M * w->ld * 4;
        if ((st = alloc((void **)&w->hi, b)) || (st = alloc((void **)&w->lo, b))) {
            free_weights(w);
            return st;
        }
        if ((st = launch(launch_split_tf32((const float *)w->main, w->ld, w->hi, w->lo, w->ld, M,
                                           K, c->stream),
                         "tf32 split (registered weights)"))) {
            free_weights(w);
            return st;
        }
    }
    if (dtype == FG_DT_INT8 && K % 4 == 0 && K >= 4 && (M / 4) * 4 > (M / 12) * 12) {
        // the reference's shifted tail rows (multigemm/src/kernel_int8.h:771-1057)
        w->tail_lo = (int)((M / 12) * 12);
        w->tail_hi = (int)((M / 4) * 4);
        w->tail_row0 = (w->tail_lo / 256) * 256;
        w->ld_tail = round_up(K + 4, 16);
        const long rows = M - w->tail_row0;
        if ((st = alloc((void **)&w->tail, (size_t)rows * w->ld_tail))) {
            free_weights(w);
            return st;
        }
        if ((st = launch(launch_prep_int8_weights((const int8_t *)w->main + (size_t)w->tail_row0 * w->ld,
                                                  w->ld, w->tail, w->ld_tail, rows, K,
                                                  w->tail_lo - w->tail_row0,
                                                  w->tail_hi - w->tail_row0, c->stream),
                         "int8 tail-row prep (registered weights)"))) {
            free_weights(w);
            return st;
        }
    }
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        free_weights(w);
        return fail(FG_ERR_CUDA, "weights: %s", cudaGetErrorString(e));
    }
    *out = w;
    return ok();
}

PreparedW prepared_of(const fg_weights_s *w)
{
    PreparedW p;
    memset(&p, 0, sizeof p);
    p.w = w->main;
    p.ld = w->ld;
    p.hi = w->hi;
    p.lo = w->lo;
    p.ld_split = w->ld;
    p.tail = w->tail;
    p.ld_tail = w->ld_tail;
    p.tail_row0 = w->tail_row0;
    p.tail_lo = w->tail_lo;
    p.tail_hi = w->tail_hi;
    return p;
}

}  // namespace

// Status setters for the library's other host files (fg_noalloc.cu).
namespace fg {
int api_fail(int status, const char *msg) { return fail(status, "%s", msg); }
int api_ok() { return ok(); }
}  // namespace fg

// ==================================================================== C ABI

FG_EXPORT int flashgemm_thread_num = 1;

FG_EXPORT void flashgemm_set_thread_num(int num) { flashgemm_thread_num = num; }

FG_EXPORT void flashgemm_multi_f32f32f32(float *C, float *B, long N, int num_gemm, ...)
{
    va_list ap;
    va_start(ap, num_gemm);
    chain_va(FG_DT_F32, C, B, N, num_gemm, ap);
    va_end(ap);
}

FG_EXPORT void flashgemm_multi_bf16bf16f32(float *C, uint16_t *B, long N, int num_gemm, ...)
{
    va_list ap;
    va_start(ap, num_gemm);
    chain_va(FG_DT_BF16, C, B, N, num_gemm, ap);
    va_end(ap);
}

FG_EXPORT void flashgemm_multi_int8uint8int32(int *C, uint8_t *B, long N, int num_gemm, ...)
{
    va_list ap;
    va_start(ap, num_gemm);
    chain_va(FG_DT_INT8, C, B, N, num_gemm, ap);
    va_end(ap);
}

FG_EXPORT void LibShalom_sgemm_mp(int transa, int transb, float *C, float *A, float *B, long M,
                                  long N, long K)
{
    (void)transa;
    if (transb == 1) {  // NT: the reference only picks a thread grid (FP32_ID23.c:39-43)
        ok();
        return;
    }
    if (transb != 0) {
        fail(FG_ERR_INVALID, "transb must be 0 or 1");
        return;
    }
    host_sgemm(C, A, B, M, N, K);
}

FG_EXPORT void LibShalom_set_thread_nums(int num) { g_shalom_threads = num; }

FG_EXPORT void Small_NGM_NN_SGEMM(float *C, float *A, float *B, long M, long N, long K, int NUM,
                                  int Tm, int Tn)
{
    (void)NUM; (void)Tm; (void)Tn;
    host_sgemm(C, A, B, M, N, K);
}

FG_EXPORT void Small_MGN_NN_SGEMM(float *C, float *A, float *B, long M, long N, long K, int NUM,
                                  int Tm, int Tn)
{
    (void)NUM; (void)Tm; (void)Tn;
    host_sgemm(C, A, B, M, N, K);
}

// C++-linkage (mangled) names of the singlegemm entry points, which is how the
// reference's g++-compiled callers reference them (singlegemm/FP32_ID23.c:35,
// set_TmTn.h:61, NN_mp.h:11 and :245).
#define FG_CXX_ALIAS(decl, mangled) __attribute__((visibility("default"))) decl __asm__(mangled)
FG_CXX_ALIAS(void fg_cxx_sgemm_mp(int, int, float *, float *, float *, long, long, long),
             "_Z18LibShalom_sgemm_mpiiPfS_S_lll");
FG_CXX_ALIAS(void fg_cxx_set_thread_nums(int), "_Z25LibShalom_set_thread_numsi");
FG_CXX_ALIAS(void fg_cxx_ngm(float *, float *, float *, long, long, long, int, int, int),
             "_Z18Small_NGM_NN_SGEMMPfS_S_llliii");
FG_CXX_ALIAS(void fg_cxx_mgn(float *, float *, float *, long, long, long, int, int, int),
             "_Z18Small_MGN_NN_SGEMMPfS_S_llliii");
void fg_cxx_sgemm_mp(int ta, int tb, float *C, float *A, float *B, long M, long N, long K)
{
    LibShalom_sgemm_mp(ta, tb, C, A, B, M, N, K);
}
void fg_cxx_set_thread_nums(int n) { LibShalom_set_thread_nums(n); }
void fg_cxx_ngm(float *C, float *A, float *B, long M, long N, long K, int u, int tm, int tn)
{
    Small_NGM_NN_SGEMM(C, A, B, M, N, K, u, tm, tn);
}
void fg_cxx_mgn(float *C, float *A, float *B, long M, long N, long K, int u, int tm, int tn)
{
    Small_MGN_NN_SGEMM(C, A, B, M, N, K, u, tm, tn);
}

FG_EXPORT int fg_last_status(void) { return t_status; }
FG_EXPORT const char *fg_last_error(void) { return t_msg; }
FG_EXPORT void fg_set_semantics(int sem) { g_sem.store(sem == FG_SEM_MATH ? FG_SEM_MATH : FG_SEM_REF); }
FG_EXPORT int fg_get_semantics(void) { return semantics(); }
FG_EXPORT void fg_set_f32_algo(int a) { g_f32.store(a == FG_F32_FFMA ? FG_F32_FFMA : FG_F32_3XTF32); }
FG_EXPORT int fg_get_f32_algo(void) { return f32_algo(); }
FG_EXPORT void fg_set_sgemm_algo(int a) { g_sgemm.store(a == FG_F32_3XTF32 ? FG_F32_3XTF32 : FG_F32_FFMA); }
FG_EXPORT int fg_get_sgemm_algo(void) { return sgemm_algo(); }
FG_EXPORT void fg_set_chain_mode(int mode)
{
    g_chain_mode.store(mode == FG_CHAIN_PER_GEMM ? FG_CHAIN_PER_GEMM : FG_CHAIN_FUSED);
}
FG_EXPORT int fg_get_chain_mode(void) { return fused_enabled() ? FG_CHAIN_FUSED : FG_CHAIN_PER_GEMM; }
FG_EXPORT unsigned long long fg_kernel_launches(void) { return g_launches.load(); }
FG_EXPORT const char *fg_version(void) { return "flashgemm-b200 0.1 (sm_100a)"; }

FG_EXPORT int fg_chain_dev(int dtype, void *C, const void *B, long N, int num_gemm,
                           const void *const *A, const long *M, const long *K, void *stream)
{
    if (dtype != FG_DT_F32 && dtype != FG_DT_BF16 && dtype != FG_DT_INT8)
        return fail(FG_ERR_INVALID, "unknown dtype %d", dtype);
    if (!C || !B || !A || !M || !K) return fail(FG_ERR_INVALID, "null pointer");
    int st = check_shapes(dtype, N, num_gemm, M, K);
    if (st) return st;
    for (int i = 0; i < num_gemm; ++i)
        if (K[i] % 2 != 0) return fail(FG_ERR_INVALID, "gemm %d: K must be a multiple of 2", i + 1);
    if (N == 0) return ok();
    const int elt = elt_of(dtype);
    if (!aligned16(C) || !aligned16(B))
        return fail(FG_ERR_INVALID, "device pointers must be 16-byte aligned");
    for (int i = 0; i < num_gemm; ++i)
        if (!A[i]) return fail(FG_ERR_INVALID, "null weight pointer");
    DevCtx *c;
    if ((st = get_ctx(&c))) return st;
    std::lock_guard<std::mutex> lk(c->mu);
    const int algo = f32_algo();
    const long ldN = round_up(N, 16);
    // B needs 16-byte rows for the tensor path; otherwise it is staged padded
    const bool tensor = !(dtype == FG_DT_F32 && algo == FG_F32_FFMA);
    const bool pad_b = tensor && ((N * elt) % 16 != 0);
    size_t need = chain_scratch(dtype, algo, N, num_gemm, M, K) + 4096;
    if (pad_b) need += carve_size((size_t)K[0] * ldN * elt);
    if ((st = arena_reserve(c, need))) return st;
    if ((st = fence_in(c, stream))) return st;
    Mat b{B, N};
    if (pad_b) {
        void *p = arena_take(c, (size_t)K[0] * ldN * elt);
        CUDA_TRY(cudaMemcpy2DAsync(p, ldN * elt, B, N * elt, N * elt, K[0], cudaMemcpyDeviceToDevice,
                                   c->stream));
        b = Mat{p, ldN};
    }
    std::vector<Mat> a(num_gemm);
    for (int i = 0; i < num_gemm; ++i) a[i] = Mat{A[i], K[i]};
    if ((st = run_chain(c, dtype, semantics(), algo, C, N, b, N, num_gemm, a.data(), M, K)))
        return st;
    if ((st = fence_out(c, stream))) return st;
    return ok();
}

FG_EXPORT int fg_sgemm_dev(float *C, const float *A, const float *B, long M, long N, long K,
                           int algo, void *stream)
{
    if (!C || !A || !B) return fail(FG_ERR_INVALID, "null pointer");
    if (M < 0 || N < 0 || K < 0) return fail(FG_ERR_INVALID, "negative dimension");
    if (M == 0 || N == 0) return ok();
    if (algo != FG_F32_FFMA && algo != FG_F32_3XTF32) return fail(FG_ERR_INVALID, "unknown algo");
    if (algo == FG_F32_3XTF32 && (K == 0 || (N % 4) || !aligned16(B) || !aligned16(C)))
        return fail(FG_ERR_UNSUPPORTED, "3xTF32 needs K > 0, N %% 4 == 0 and 16-byte-aligned B, C");
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    std::lock_guard<std::mutex> lk(c->mu);
    size_t need = 4096;
    if (algo == FG_F32_3XTF32) {
        long Ms[1] = {M}, Ks[1] = {K};
        need += chain_scratch(FG_DT_F32, algo, N, 1, Ms, Ks);
    }
    if ((st = arena_reserve(c, need))) return st;
    if ((st = fence_in(c, stream))) return st;
    if ((st = run_sgemm(c, algo, C, N, A, K, B, N, M, N, K, 2048))) return st;
    if ((st = fence_out(c, stream))) return st;
    return ok();
}

FG_EXPORT int fg_sync(void)
{
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    std::lock_guard<std::mutex> lk(c->mu);
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if ((st = collect_status(c))) return st;
    return ok();
}

FG_EXPORT int fg_profile_begin(void)
{
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    std::lock_guard<std::mutex> lk(c->mu);
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (auto &r : c->prof) c->prof_pool.push_back(r);
    c->prof.clear();
    g_prof_on.store(1);
    return ok();
}

FG_EXPORT int fg_profile_end(void)
{
    g_prof_on.store(0);
    return ok();
}

FG_EXPORT int fg_profile_query(int kind, double *total_ms, unsigned long long *launches,
                               double *flops)
{
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    std::lock_guard<std::mutex> lk(c->mu);
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    double ms = 0.0, fl = 0.0;
    unsigned long long n = 0;
    for (auto &r : c->prof) {
        if (kind >= 0 && r.kind != kind) continue;
        float t = 0.f;
        CUDA_TRY(cudaEventElapsedTime(&t, r.a, r.b));
        ms += t;
        fl += r.flops;
        ++n;
    }
    if (total_ms) *total_ms = ms;
    if (launches) *launches = n;
    if (flops) *flops = fl;
    return ok();
}

FG_EXPORT int fg_weights_register(int dtype, const void *A, long M, long K, int where,
                                  fg_weights *out)
{
    return register_weights(dtype, A, M, K, where, out);
}

FG_EXPORT int fg_weights_release(fg_weights w)
{
    if (!w) return ok();
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != w->dev) cudaSetDevice(w->dev);
    cudaDeviceSynchronize();  // no chain may still read them
    free_weights(w);
    if (cur != w->dev) cudaSetDevice(cur);
    return ok();
}

FG_EXPORT long fg_weights_bytes(fg_weights w) { return w ? (long)w->bytes : 0; }

FG_EXPORT int fg_chain_registered(int dtype, void *C, const void *B, long N, int num_gemm,
                                  const fg_weights *W, void *stream)
{
    if (!C || !B || !W) return fail(FG_ERR_INVALID, "null pointer");
    if (num_gemm < 1 || num_gemm > 4096) return fail(FG_ERR_INVALID, "num_gemm out of range");
    std::vector<long> M(num_gemm), K(num_gemm);
    std::vector<PreparedW> pw(num_gemm);
    std::vector<Mat> a(num_gemm);
    for (int i = 0; i < num_gemm; ++i) {
        if (!W[i]) return fail(FG_ERR_INVALID, "null weight handle");
        if (W[i]->dtype != dtype) return fail(FG_ERR_INVALID, "gemm %d: weights of another dtype", i + 1);
        M[i] = W[i]->M;
        K[i] = W[i]->K;
        pw[i] = prepared_of(W[i]);
        a[i] = Mat{W[i]->main, W[i]->ld};
    }
    int st = check_shapes(dtype, N, num_gemm, M.data(), K.data());
    if (st) return st;
    for (int i = 0; i < num_gemm; ++i)
        if (K[i] % 2 != 0) return fail(FG_ERR_INVALID, "gemm %d: K must be a multiple of 2", i + 1);
    if (N == 0) return ok();
    if (!aligned16(C) || !aligned16(B))
        return fail(FG_ERR_INVALID, "device pointers must be 16-byte aligned");
    DevCtx *c;
    if ((st = get_ctx(&c))) return st;
    for (int i = 0; i < num_gemm; ++i)
        if (W[i]->dev != c->dev)
            return fail(FG_ERR_INVALID, "gemm %d: weights registered on device %d", i + 1, W[i]->dev);
    std::lock_guard<std::mutex> lk(c->mu);
    const int elt = elt_of(dtype);
    const int algo = f32_algo();
    const long ldN = round_up(N, 16);
    const bool tensor = !(dtype == FG_DT_F32 && algo == FG_F32_FFMA);
    const bool pad_b = tensor && ((N * elt) % 16 != 0);
    size_t need = chain_scratch(dtype, algo, N, num_gemm, M.data(), K.data()) + 4096;
    if (pad_b) need += carve_size((size_t)K[0] * ldN * elt);
    if ((st = arena_reserve(c, need))) return st;
    if ((st = fence_in(c, stream))) return st;
    Mat b{B, N};
    if (pad_b) {
        void *p = arena_take(c, (size_t)K[0] * ldN * elt);
        CUDA_TRY(cudaMemcpy2DAsync(p, ldN * elt, B, N * elt, N * elt, K[0], cudaMemcpyDeviceToDevice,
                                   c->stream));
        b = Mat{p, ldN};
    }
    if ((st = run_chain(c, dtype, semantics(), algo, C, N, b, N, num_gemm, a.data(), M.data(),
                        K.data(), pw.data())))
        return st;
    if ((st = fence_out(c, stream))) return st;
    return ok();
}

// ---------------------------------------------------------------- grouped launches

namespace {

// Device bytes of one chain's between-stage buffers in a grouped launch
// (registered weights need no copies).
size_t group_chain_bytes(int dtype, int algo, long N, int n, const long *M, const long *K)
{
    const long ldN = round_up(N, 16);
    long maxM = 0;
    for (int i = 0; i < n - 1; ++i) maxM = M[i] > maxM ? M[i] : maxM;
    const bool x3 = dtype == FG_DT_F32 && algo == FG_F32_3XTF32;
    size_t s = 1024;
    if (n > 1) s += (x3 ? 4 : 2) * carve_size((size_t)maxM * ldN * elt_of(dtype));
    if (x3) s += 2 * carve_size((size_t)K[0] * ldN * 4);  // split activations
    return s;
}

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
    int kernels() const
    {
        return (int)gls.size() + (splits.empty() ? 0 : 1) + (int)levels.size();
    }
};

int group_check(DevCtx *c, int dtype, int nchains, const fg_chain_desc *chains)
{
    if (nchains < 1 || !chains) return fail(FG_ERR_INVALID, "no chains");
    if (dtype != FG_DT_BF16 && dtype != FG_DT_INT8 && dtype != FG_DT_F32)
        return fail(FG_ERR_INVALID, "unknown dtype %d", dtype);
    const int elt = elt_of(dtype);
    for (int j = 0; j < nchains; ++j) {
        const fg_chain_desc &d = chains[j];
        if (!d.C || !d.B || !d.W || d.num_gemm < 1 || d.num_gemm > 4096)
            return fail(FG_ERR_INVALID, "chain %d: null pointer or bad GEMM count", j);
        if (d.N <= 0 || d.N > (1l << 30) || (d.N * elt) % 16)
            return fail(FG_ERR_INVALID, "chain %d: N must be positive with 16-byte rows", j);
        if (!aligned16(d.C) || !aligned16(d.B))
            return fail(FG_ERR_INVALID, "chain %d: pointers must be 16-byte aligned", j);
        for (int i = 0; i < d.num_gemm; ++i) {
            if (!d.W[i] || d.W[i]->dtype != dtype)
                return fail(FG_ERR_INVALID, "chain %d gemm %d: weights missing or of another dtype",
                            j, i + 1);
            if (d.W[i]->dev != c->dev)
                return fail(FG_ERR_INVALID, "chain %d gemm %d: weights registered on device %d", j,
                            i + 1, d.W[i]->dev);
            if (i > 0 && d.W[i]->K != d.W[i - 1]->M)
                return fail(FG_ERR_INVALID, "chain %d gemm %d: K must equal the previous M", j,
                            i + 1);
            if (d.W[i]->K % 2) return fail(FG_ERR_INVALID, "chain %d: K must be even", j);
        }
    }
    return FG_OK;
}

size_t group_buf_bytes(int dtype, int algo, int nchains, const fg_chain_desc *chains)
{
    size_t need = 4096;
    for (int j = 0; j < nchains; ++j) {
        const fg_chain_desc &d = chains[j];
        std::vector<long> M(d.num_gemm), K(d.num_gemm);
        for (int i = 0; i < d.num_gemm; ++i) {
            M[i] = d.W[i]->M;
            K[i] = d.W[i]->K;
        }
        need += group_chain_bytes(dtype, algo, d.N, d.num_gemm, M.data(), K.data());
    }
    return need;
}

// Cost model of a grouped launch (microseconds), closed form so that it costs
// far less than the launch it chooses for. A tile takes the longer of its MMA
// time (k-blocks x one k-block on the tile's SMs at the measured dense BF16
// rate per SM; INT8 k-blocks hold twice the K at twice the rate, TF32 runs at
// half the rate and 3xTF32 issues three MMAs) and its epilogue (output bytes
// per SM at about 16 GB/s per SM, the staged drain's measured rate), plus
// 0.3 us. Levels: each level takes max(its work / workers, its longest tile)
// plus 3 us of launch; fused: max(all work / workers, the longest chain's
// tiles back to back with 2 us hand-offs). The result is divided by the
// kernel's efficiency measured on the 512-chain grouped workload relative to
// the best kernel for that operand type (B200: BF16 pair 0.98, 128x256 1.0,
// 128x128 0.77; INT8 pair 0.85, 128x256 1.0, 128x128 0.80). Fused runs of the
// pair kernel, whose CTA pairs follow static lists, pay the 10% their
// dependency waits cost there; the single-CTA kernel takes its tiles from one
// list in turn and pays none.
struct ModelStage {
    long M, N, K;
    int prev, depth;
};

double model_makespan(int kernel, int order, int op, int sms, const std::vector<ModelStage> &st)
{
    const bool pair = op != OP_TF32X3 && kernel == GK_PAIR;
    const double units = pair ? sms / 2 : sms;
    const double tm = pair ? 256 : 128, tn = pair ? 256 : group_tile_n(kernel, op);
    const double sm_per_tile = pair ? 2.0 : 1.0;
    const double kb_elems = op == OP_I8 ? 128.0 : op == OP_BF16 ? 64.0 : 32.0;
    const double rate = 1600.0 / 148.0 * sm_per_tile *
                        (op == OP_I8 ? 2.0 : op == OP_TF32X3 ? 0.5 / 3.0 : 1.0);  // TFLOP/s
    const double t_kb = 2.0 * tm * tn * kb_elems / (rate * 1e6);
    const double out_elt = op == OP_I8 ? 1.0 : op == OP_BF16 ? 2.0 : 8.0;
    const double t_epi = tm * tn * out_elt / sm_per_tile / 16e3;
    std::vector<double> tile(st.size()), work(st.size());
    int maxd = 0;
    for (size_t i = 0; i < st.size(); ++i) {
        const double kb = std::ceil((double)st[i].K / kb_elems);
        tile[i] = std::max(kb * t_kb, t_epi) + 0.3;
        work[i] = tile[i] * std::ceil(st[i].M / tm) * std::ceil(st[i].N / tn);
        maxd = std::max(maxd, st[i].depth);
    }
    double eff = 1.0;
    if (op == OP_BF16) eff = kernel == GK_PAIR ? 0.98 : kernel == GK_SINGLE_256 ? 1.0 : 0.77;
    if (op == OP_I8) eff = kernel == GK_PAIR ? 0.85 : kernel == GK_SINGLE_256 ? 1.0 : 0.80;
    double t = 0.0;
    if (order == FG_ORDER_LEVELS) {
        std::vector<double> lw(maxd + 1, 0.0), lt(maxd + 1, 0.0);
        for (size_t i = 0; i < st.size(); ++i) {
            lw[st[i].depth] += work[i];
            lt[st[i].depth] = std::max(lt[st[i].depth], tile[i]);
        }
        for (int l = 0; l <= maxd; ++l) t += std::max(lw[l] / units, lt[l]) + 3.0;
    } else {
        double total = 0.0, crit = 0.0;
        std::vector<double> path(st.size(), 0.0);
        for (size_t i = 0; i < st.size(); ++i) {
            total += work[i];
            path[i] = (st[i].prev >= 0 ? path[st[i].prev] + 2.0 : 0.0) + tile[i];
            crit = std::max(crit, path[i]);
        }
        t = std::max((pair ? 1.10 : 1.0) * total / units, crit) + 3.0;
    }
    return t / eff;
}

// ---------------------------------------------------------------- autotuner memory

std::mutex g_tune_mu;
std::vector<std::pair<std::string, std::pair<int, int>>> g_tune;  // signature -> (kernel, order)
std::atomic<int> g_group_kernel{FG_GROUP_AUTO}, g_group_order{FG_ORDER_AUTO};

// Shape signature of a group: dtype, FP32 algorithm and the sorted chain shapes.
std::string group_signature(int dtype, int algo, int nchains, const fg_chain_desc *chains)
{
    std::vector<std::string> parts;
    for (int j = 0; j < nchains; ++j) {
        std::string p = std::to_string(chains[j].N);
        for (int i = 0; i < chains[j].num_gemm; ++i)
            p += (i ? "," : ":") + std::to_string(chains[j].W[i]->M) + "x" +
                 std::to_string(chains[j].W[i]->K);
        parts.push_back(p);
    }
    std::sort(parts.begin(), parts.end());
    std::string s = std::to_string(dtype) + "/" + std::to_string(algo);
    for (auto &p : parts) s += ";" + p;
    return s;
}

bool tune_lookup(const std::string &sig, int &kernel, int &order)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (auto &e : g_tune)
        if (e.first == sig) {
            kernel = e.second.first;
            order = e.second.second;
            return true;
        }
    return false;
}

void tune_store(const std::string &sig, int kernel, int order)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (auto &e : g_tune)
        if (e.first == sig) {
            e.second = {kernel, order};
            return;
        }
    g_tune.push_back({sig, {kernel, order}});
}

// Resolves FG_GROUP_AUTO / FG_ORDER_AUTO: remembered measurement, else the model.
void group_resolve(DevCtx *c, int dtype, int algo, int nchains, const fg_chain_desc *chains,
                   int &kernel, int &order)
{
    if (dtype == FG_DT_F32 && algo == FG_F32_FFMA) {
        kernel = GK_SINGLE_128;  // not used: the CUDA-core path runs one launch per depth
        order = FG_ORDER_LEVELS;
        return;
    }
    const int op = dtype == FG_DT_BF16 ? OP_BF16 : dtype == FG_DT_INT8 ? OP_I8 : OP_TF32X3;
    if (op == OP_TF32X3) kernel = GK_SINGLE_128;
    if (kernel != FG_GROUP_AUTO && order != FG_ORDER_AUTO) return;
    int tk = 0, to = 0;
    if (tune_lookup(group_signature(dtype, algo, nchains, chains), tk, to)) {
        if (kernel == FG_GROUP_AUTO) kernel = tk;
        if (order == FG_ORDER_AUTO) order = to;
        if (op == OP_TF32X3) kernel = GK_SINGLE_128;
        return;
    }
    std::vector<ModelStage> st;
    for (int j = 0; j < nchains; ++j)
        for (int i = 0; i < chains[j].num_gemm; ++i)
            st.push_back(ModelStage{chains[j].W[i]->M, chains[j].N, chains[j].W[i]->K,
                                    i == 0 ? -1 : (int)st.size() - 1, i});
    double best = 1e300;
    int bk = GK_PAIR, bo = FG_ORDER_FUSED;
    const int kmin = op == OP_TF32X3 ? GK_SINGLE_128 : GK_PAIR;
    for (int k = kmin; k <= GK_SINGLE_128; ++k) {
        if (kernel != FG_GROUP_AUTO && k != kernel) continue;
        for (int o = FG_ORDER_FUSED; o <= FG_ORDER_LEVELS; ++o) {
            if (order != FG_ORDER_AUTO && o != order) continue;
            const double t = model_makespan(k, o, op, c->sms, st);
            if (t < best - 1e-9) best = t, bk = k, bo = o;
        }
    }
    kernel = bk;
    order = bo;
}

// Host side of a grouped launch: between-stage buffers carved from `cv`, stage
// lists, schedules and tables (device addresses of the tables come later).
int group_build(DevCtx *c, int dtype, int algo, int kernel, int order, int nchains,
                const fg_chain_desc *chains, Carver &cv, GroupExec &gx, int *status = nullptr,
                int max_units = 0)
{
    if (!status) status = c->status;
    gx.dtype = dtype;
    gx.algo = algo;
    gx.kernel = kernel;
    gx.order = order;
    const int sem = semantics();
    std::vector<StageArgs> all;
    std::vector<int> prev, depth;
    int maxd = 0;
    for (int j = 0; j < nchains; ++j) {
        const fg_chain_desc &d = chains[j];
        const int n = d.num_gemm;
        std::vector<long> M(n), K(n);
        std::vector<PreparedW> pw(n);
        std::vector<Mat> a(n);
        for (int i = 0; i < n; ++i) {
            M[i] = d.W[i]->M;
            K[i] = d.W[i]->K;
            pw[i] = prepared_of(d.W[i]);
            a[i] = Mat{d.W[i]->main, d.W[i]->ld};
            gx.flops += gemm_flops(M[i], d.N, K[i]);
        }
        maxd = std::max(maxd, n - 1);
        const long N = d.N, ldN = round_up(N, 16);
        long maxM = 0;
        for (int i = 0; i < n - 1; ++i) maxM = std::max(maxM, M[i]);
        if (dtype == FG_DT_F32 && algo == FG_F32_FFMA) {
            float *buf[2] = {nullptr, nullptr};
            if (n > 1)
                for (int q = 0; q < 2; ++q) buf[q] = (float *)cv.take((size_t)maxM * ldN * 4);
            const float *x = (const float *)d.B;
            long ldx = N;
            if ((int)gx.levels.size() < n) gx.levels.resize(n);
            for (int i = 0; i < n; ++i) {
                const bool last = (i == n - 1);
                FfmaJob f;
                memset(&f, 0, sizeof f);
                f.M = (int)M[i]; f.N = (int)N; f.K = (int)K[i];
                f.A = (const float *)pw[i].w; f.lda = pw[i].ld;
                f.B = x; f.ldb = ldx;
                f.C = last ? (float *)d.C : buf[i & 1];
                f.ldc = last ? N : ldN;
                f.vec = ((f.lda | f.ldb | f.ldc) % 4 == 0) &&
                        ((((uintptr_t)f.A | (uintptr_t)f.B | (uintptr_t)f.C) & 15) == 0);
                gx.levels[i].jobs.push_back(f);
                gx.levels[i].flops += gemm_flops(M[i], N, K[i]);
                x = f.C;
                ldx = f.ldc;
            }
            continue;
        }
        std::vector<StageArgs> stg;
        if (dtype == FG_DT_F32) {  // 3xTF32 on the registered hi / lo split
            float *xh = (float *)cv.take((size_t)K[0] * ldN * 4);
            float *xl = (float *)cv.take((size_t)K[0] * ldN * 4);
            gx.splits.push_back(SplitJob{(const float *)d.B, N, xh, xl, ldN, K[0], N});
            gx.split_max = std::max(gx.split_max, K[0] * N);
            float *ph[2] = {nullptr, nullptr}, *pl[2] = {nullptr, nullptr};
            if (n > 1)
                for (int q = 0; q < 2; ++q) {
                    ph[q] = (float *)cv.take((size_t)maxM * ldN * 4);
                    pl[q] = (float *)cv.take((size_t)maxM * ldN * 4);
                }
            for (int i = 0; i < n; ++i) {
                const bool last = (i == n - 1);
                StageArgs s;
                memset(&s, 0, sizeof s);
                s.status = status;
                s.op = OP_TF32X3;
                s.M = (int)M[i]; s.N = (int)N; s.K = (int)K[i];
                s.w = pw[i].hi; s.w_lo = pw[i].lo; s.ld_w = pw[i].ld_split;
                s.x = xh; s.x_lo = xl; s.ld_x = ldN;
                s.epi = last ? EPI_F32 : EPI_TF32SPLIT;
                s.out = last ? d.C : (void *)ph[i & 1];
                s.out_lo = last ? nullptr : (void *)pl[i & 1];
                s.ld_out = last ? N : ldN;
                s.m_written = (int)M[i];
                s.kchunk = tf32_chunk_blocks(K[i]);
                stg.push_back(s);
                xh = ph[i & 1];
                xl = pl[i & 1];
            }
        } else {
            int st = build_tc_stages(c, dtype, sem, d.C, N, Mat{d.B, N}, N, n, a.data(), M.data(),
                                     K.data(), pw.data(), stg, &cv);
            if (st) return st;
            for (auto &x : stg) x.status = status;
        }
        const int base = (int)all.size();
        for (int i = 0; i < n; ++i) {
            all.push_back(stg[i]);
            prev.push_back(i == 0 ? -1 : base + i - 1);
            depth.push_back(i);
        }
    }
    if (dtype == FG_DT_F32 && algo == FG_F32_FFMA) {
        for (auto &lv : gx.levels) {
            long t128 = 0;
            for (auto &f : lv.jobs) t128 += (long)((f.M + 127) / 128) * ((f.N + 127) / 128);
            lv.big = t128 >= 2l * c->sms ? 1 : 0;
            const int tile = ffma_group_tile(lv.big);
            long t = 0;
            for (auto &f : lv.jobs) {
                f.tile0 = (int)t;
                f.tiles_n = (f.N + tile - 1) / tile;
                t += (long)((f.M + tile - 1) / tile) * f.tiles_n;
            }
            if (t > (1l << 31) - 1) return fail(FG_ERR_INVALID, "group too large");
            lv.tiles = (int)t;
        }
        return FG_OK;
    }
    const int nlaunch = order == FG_ORDER_LEVELS ? maxd + 1 : 1;
    for (int lv = 0; lv < nlaunch; ++lv) {
        std::vector<StageArgs> st;
        std::vector<int> pv;
        std::vector<int> remap(all.size(), -1);
        double fl = 0.0;
        for (size_t i = 0; i < all.size(); ++i) {
            if (order == FG_ORDER_LEVELS && depth[i] != lv) continue;
            remap[i] = (int)st.size();
            pv.push_back(order == FG_ORDER_LEVELS ? -1 : (prev[i] >= 0 ? remap[prev[i]] : -1));
            st.push_back(all[i]);
            fl += gemm_flops(all[i].M, all[i].N, all[i].K);
        }
        GroupLaunch gl;
        cudaError_t e = plan_group(st.data(), pv.data(), (int)st.size(), kernel,
                                   max_units > 0 ? max_units : c->sms, gl);
        if (e != cudaSuccess)
            return fail(e == cudaErrorNotSupported ? FG_ERR_INVALID : FG_ERR_CUDA,
                        "grouped launch plan: %s", cudaGetErrorString(e));
        gx.gls.push_back(std::move(gl));
        gx.gl_flops.push_back(fl);
    }
    return FG_OK;
}

size_t group_tab_bytes(const GroupExec &gx)
{
    size_t b = 4096;
    size_t done = 0;
    for (auto &gl : gx.gls) {
        b += carve_size(gl.tables.size());
        done += gl.done_ints;
    }
    b += carve_size(done * sizeof(int) + 16);
    b += carve_size(gx.splits.size() * sizeof(SplitJob));
    for (auto &lv : gx.levels) b += carve_size(lv.jobs.size() * sizeof(FfmaJob));
    return b;
}

// Device addresses of the tables, counters and job lists.
void group_place(GroupExec &gx, Carver &cv)
{
    gx.tables.clear();
    gx.done_at.clear();
    gx.done_ints = 0;
    for (auto &gl : gx.gls) {
        gx.tables.push_back(cv.take(gl.tables.size()));
        gx.done_at.push_back(gx.done_ints);
        gx.done_ints += gl.done_ints;
    }
    gx.done = (int *)cv.take(gx.done_ints * sizeof(int) + 16);
    gx.splits_dev = gx.splits.empty() ? nullptr
                                      : (SplitJob *)cv.take(gx.splits.size() * sizeof(SplitJob));
    for (auto &lv : gx.levels) lv.dev = (FfmaJob *)cv.take(lv.jobs.size() * sizeof(FfmaJob));
}

int group_upload(const GroupExec &gx, cudaStream_t s, bool sync)
{
    auto copy = [&](void *dst, const void *src, size_t bytes) -> cudaError_t {
        if (!bytes) return cudaSuccess;
        return sync ? cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice)
                    : cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
    };
    for (size_t i = 0; i < gx.gls.size(); ++i)
        CUDA_TRY(copy(gx.tables[i], gx.gls[i].tables.data(), gx.gls[i].tables.size()));
    CUDA_TRY(copy(gx.splits_dev, gx.splits.data(), gx.splits.size() * sizeof(SplitJob)));
    for (auto &lv : gx.levels) CUDA_TRY(copy(lv.dev, lv.jobs.data(), lv.jobs.size() * sizeof(FfmaJob)));
    return FG_OK;
}

int group_launch(DevCtx *c, const GroupExec &gx, cudaStream_t s, bool capturing,
                 int *status = nullptr)
{
    if (!status) status = c->status;
    if (gx.done_ints) CUDA_TRY(cudaMemsetAsync(gx.done, 0, gx.done_ints * sizeof(int), s));
    if (!gx.splits.empty()) {
        int st = run_kernel_on(c, s, capturing, FG_PK_AUX, 0.0, "tf32 split (group)", [&] {
            return launch_split_tf32_jobs(gx.splits_dev, (int)gx.splits.size(), gx.split_max, s);
        });
        if (st) return st;
    }
    const int kind = gx.dtype == FG_DT_BF16 ? FG_PK_TC_BF16
                   : gx.dtype == FG_DT_INT8 ? FG_PK_TC_I8
                                            : FG_PK_TC_TF32X3;
    for (size_t i = 0; i < gx.gls.size(); ++i) {
        int st = run_kernel_on(c, s, capturing, kind, gx.gl_flops[i], "grouped chains", [&] {
            return launch_group(gx.gls[i], gx.tables[i], gx.done + gx.done_at[i], status, s);
        });
        if (st) return st;
    }
    for (auto &lv : gx.levels) {
        int st = run_kernel_on(c, s, capturing, FG_PK_FFMA, lv.flops, "grouped ffma", [&] {
            return launch_ffma_group(lv.dev, (int)lv.jobs.size(), lv.tiles, lv.big, s);
        });
        if (st) return st;
    }
    return FG_OK;
}

}  // namespace

struct fg_plan_s {
    int dev = -1;
    GroupExec gx;
    void *buf = nullptr, *tab = nullptr;
    size_t bytes = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

void plan_free(fg_plan_s *p)
{
    if (!p) return;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    cudaFree(p->buf);
    cudaFree(p->tab);
    delete p;
}

// A plan with its own device memory; the caller holds c->mu.
int plan_make(DevCtx *c, int dtype, int algo, int kernel, int order, int nchains,
              const fg_chain_desc *chains, fg_plan_s **out)
{
    fg_plan_s *p = new fg_plan_s;
    p->dev = c->dev;
    const size_t nb = group_buf_bytes(dtype, algo, nchains, chains);
    cudaError_t e = cudaMalloc(&p->buf, nb);
    if (e != cudaSuccess) {
        cudaGetLastError();
        plan_free(p);
        return fail(FG_ERR_NOMEM, "plan buffers of %zu bytes: %s", nb, cudaGetErrorString(e));
    }
    Carver cb;
    cb.base = (char *)p->buf;
    int st = group_build(c, dtype, algo, kernel, order, nchains, chains, cb, p->gx);
    if (st) {
        plan_free(p);
        return st;
    }
    const size_t tb = group_tab_bytes(p->gx);
    e = cudaMalloc(&p->tab, tb);
    if (e != cudaSuccess) {
        cudaGetLastError();
        plan_free(p);
        return fail(FG_ERR_NOMEM, "plan tables of %zu bytes: %s", tb, cudaGetErrorString(e));
    }
    Carver ct;
    ct.base = (char *)p->tab;
    group_place(p->gx, ct);
    if ((st = group_upload(p->gx, nullptr, true))) {
        plan_free(p);
        return st;
    }
    p->bytes = nb + tb;
    *out = p;
    return FG_OK;
}

int resolved_config(DevCtx *c, int dtype, int algo, int nchains, const fg_chain_desc *chains,
                    int &kernel, int &order)
{
    kernel = g_group_kernel.load();
    order = g_group_order.load();
    group_resolve(c, dtype, algo, nchains, chains, kernel, order);
    return FG_OK;
}

}  // namespace

// Many chains of one dtype on registered weights in one grouped launch.
FG_EXPORT int fg_chain_group(int dtype, int nchains, const fg_chain_desc *chains, void *stream)
{
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    if ((st = group_check(c, dtype, nchains, chains))) return st;
    std::lock_guard<std::mutex> lk(c->mu);
    const int algo = dtype == FG_DT_F32 ? f32_algo() : 0;
    int kernel, order;
    resolved_config(c, dtype, algo, nchains, chains, kernel, order);
    if ((st = arena_reserve(c, group_buf_bytes(dtype, algo, nchains, chains)))) return st;
    Carver cb;
    cb.base = c->arena;
    GroupExec gx;
    if ((st = group_build(c, dtype, algo, kernel, order, nchains, chains, cb, gx))) return st;
    if ((st = tab_reserve(c, group_tab_bytes(gx)))) return st;
    Carver ct;
    ct.base = c->tab;
    group_place(gx, ct);
    if ((st = fence_in(c, stream))) return st;
    if ((st = group_upload(gx, c->stream, false))) return st;
    if ((st = group_launch(c, gx, c->stream, false))) return st;
    if ((st = fence_out(c, stream))) return st;
    return ok();
}

FG_EXPORT void fg_set_group_config(int kernel, int order)
{
    g_group_kernel.store(kernel >= FG_GROUP_PAIR && kernel <= FG_GROUP_SINGLE_128 ? kernel
                                                                                  : FG_GROUP_AUTO);
    g_group_order.store(order == FG_ORDER_FUSED || order == FG_ORDER_LEVELS ? order : FG_ORDER_AUTO);
}

FG_EXPORT void fg_get_group_config(int *kernel, int *order)
{
    if (kernel) *kernel = g_group_kernel.load();
    if (order) *order = g_group_order.load();
}

FG_EXPORT int fg_group_choice(int dtype, int nchains, const fg_chain_desc *chains, int *kernel,
                              int *order)
{
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    if ((st = group_check(c, dtype, nchains, chains))) return st;
    const int algo = dtype == FG_DT_F32 ? f32_algo() : 0;
    int k, o;
    resolved_config(c, dtype, algo, nchains, chains, k, o);
    if (kernel) *kernel = k;
    if (order) *order = o;
    return ok();
}

FG_EXPORT int fg_plan_create(int dtype, int nchains, const fg_chain_desc *chains, fg_plan *out)
{
    if (!out) return fail(FG_ERR_INVALID, "null plan pointer");
    *out = nullptr;
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    if ((st = group_check(c, dtype, nchains, chains))) return st;
    std::lock_guard<std::mutex> lk(c->mu);
    const int algo = dtype == FG_DT_F32 ? f32_algo() : 0;
    int kernel, order;
    resolved_config(c, dtype, algo, nchains, chains, kernel, order);
    fg_plan_s *p = nullptr;
    if ((st = plan_make(c, dtype, algo, kernel, order, nchains, chains, &p))) return st;
    *out = p;
    return ok();
}

FG_EXPORT int fg_plan_launch(fg_plan plan, void *stream)
{
    if (!plan) return fail(FG_ERR_INVALID, "null plan");
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    if (plan->dev != c->dev) return fail(FG_ERR_INVALID, "plan belongs to device %d", plan->dev);
    std::lock_guard<std::mutex> lk(c->mu);
    cudaStream_t s = stream ? (cudaStream_t)stream : cudaStreamLegacy;
    if ((st = group_launch(c, plan->gx, s, false))) return st;
    return ok();
}

FG_EXPORT int fg_plan_launch_graph(fg_plan plan, void *stream)
{
    if (!plan) return fail(FG_ERR_INVALID, "null plan");
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    if (plan->dev != c->dev) return fail(FG_ERR_INVALID, "plan belongs to device %d", plan->dev);
    std::lock_guard<std::mutex> lk(c->mu);
    if (!plan->exec) {
        cudaStream_t cap;
        CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            st = group_launch(c, plan->gx, cap, true);
            cudaGraph_t g = nullptr;
            e = cudaStreamEndCapture(cap, &g);
            // the captured kernels were counted as launches: they run with the graph
            g_launches.fetch_sub((unsigned long long)plan->gx.kernels(), std::memory_order_relaxed);
            if (!st && e == cudaSuccess) {
                plan->graph = g;
                e = cudaGraphInstantiate(&plan->exec, g, 0);
            } else if (g) {
                cudaGraphDestroy(g);
            }
        }
        cudaStreamDestroy(cap);
        if (st) return st;
        if (e != cudaSuccess) {
            cudaGetLastError();
            plan->exec = nullptr;
            return fail(FG_ERR_CUDA, "graph capture of the plan: %s", cudaGetErrorString(e));
        }
    }
    cudaStream_t s = stream ? (cudaStream_t)stream : cudaStreamLegacy;
    CUDA_TRY(cudaGraphLaunch(plan->exec, s));
    g_launches.fetch_add((unsigned long long)plan->gx.kernels(), std::memory_order_relaxed);
    return ok();
}

FG_EXPORT int fg_plan_info(fg_plan plan, int *kernel, int *order, long *device_bytes, int *kernels,
                           double *flops)
{
    if (!plan) return fail(FG_ERR_INVALID, "null plan");
    const bool ffma = plan->gx.dtype == FG_DT_F32 && plan->gx.algo == FG_F32_FFMA;
    if (kernel) *kernel = ffma ? -1 : plan->gx.kernel;
    if (order) *order = plan->gx.order;
    if (device_bytes) *device_bytes = (long)plan->bytes;
    if (kernels) *kernels = plan->gx.kernels();
    if (flops) *flops = plan->gx.flops;
    return ok();
}

FG_EXPORT int fg_plan_release(fg_plan plan)
{
    if (!plan) return ok();
    cudaDeviceSynchronize();
    plan_free(plan);
    return ok();
}

FG_EXPORT int fg_autotune_group(int dtype, int nchains, const fg_chain_desc *chains, int iters,
                                int *kernel, int *order, double *best_ms)
{
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    if ((st = group_check(c, dtype, nchains, chains))) return st;
    if (iters < 1) iters = 1;
    std::lock_guard<std::mutex> lk(c->mu);
    const int algo = dtype == FG_DT_F32 ? f32_algo() : 0;
    const bool ffma = dtype == FG_DT_F32 && algo == FG_F32_FFMA;
    const int kmin = dtype == FG_DT_F32 ? GK_SINGLE_128 : GK_PAIR;
    cudaStream_t s;
    CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e300;
    int bk = kmin, bo = FG_ORDER_FUSED;
    for (int k = kmin; k <= GK_SINGLE_128 && !st; ++k)
        for (int o = ffma ? FG_ORDER_LEVELS : FG_ORDER_FUSED; o <= FG_ORDER_LEVELS && !st; ++o) {
            fg_plan_s *p = nullptr;
            if ((st = plan_make(c, dtype, algo, k, o, nchains, chains, &p))) break;
            st = group_launch(c, p->gx, s, false);  // warm-up
            if (!st) cudaEventRecord(e0, s);
            for (int it = 0; it < iters && !st; ++it) st = group_launch(c, p->gx, s, false);
            if (!st) cudaEventRecord(e1, s);
            cudaError_t e = cudaStreamSynchronize(s);
            if (!st && e != cudaSuccess) st = fail(FG_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
            float ms = 0.f;
            if (!st) cudaEventElapsedTime(&ms, e0, e1);
            plan_free(p);
            if (st) break;
            const double t = ms / iters;
            if (t < best) best = t, bk = k, bo = o;
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    if (st) return st;
    if ((st = collect_status(c))) return st;
    tune_store(group_signature(dtype, algo, nchains, chains), bk, bo);
    if (kernel) *kernel = ffma ? -1 : bk;
    if (order) *order = bo;
    if (best_ms) *best_ms = best;
    return ok();
}

FG_EXPORT int fg_autotune_save(const char *path)
{
    if (!path) return fail(FG_ERR_INVALID, "null path");
    FILE *f = fopen(path, "w");
    if (!f) return fail(FG_ERR_INVALID, "cannot write %s", path);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (auto &e : g_tune) fprintf(f, "%d %d %s\n", e.second.first, e.second.second, e.first.c_str());
    fclose(f);
    return ok();
}

FG_EXPORT int fg_autotune_load(const char *path)
{
    if (!path) return fail(FG_ERR_INVALID, "null path");
    FILE *f = fopen(path, "r");
    if (!f) return fail(FG_ERR_INVALID, "cannot read %s", path);
    std::vector<char> line(1 << 20);
    int n = 0;
    while (fgets(line.data(), (int)line.size(), f)) {
        int k, o, used = 0;
        if (sscanf(line.data(), "%d %d %n", &k, &o, &used) < 2 || used <= 0) continue;
        std::string sig(line.data() + used);
        while (!sig.empty() && (sig.back() == '\n' || sig.back() == '\r')) sig.pop_back();
        if (k < GK_PAIR || k > GK_SINGLE_128 || o < FG_ORDER_FUSED || o > FG_ORDER_LEVELS) continue;
        tune_store(sig, k, o);
        ++n;
    }
    fclose(f);
    return ok();
}

// ---------------------------------------------------------------- serving loop

struct fg_server_s {
    struct Req {
        fg_request r;
        std::vector<fg_weights> W;  // the request's weight handles (copied at submit)
        long long id = 0;
        double t_submit = 0.0;
        size_t bytes = 0;           // admission estimate
        double flops = 0.0;
        bool done = false;
        int status = FG_OK;
        double latency_us = 0.0;
    };
    struct Batch {
        std::vector<Req *> reqs;
        std::vector<GroupExec> gx;  // host tables, kept until the batch completes
        int slot = 0;
        size_t bytes = 0;
        void *mem = nullptr, *tab = nullptr;
        int status = FG_OK;
    };

    DevCtx *c = nullptr;
    fg_server_opts o{};
    cudaMemPool_t pool = nullptr;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> events;
    int *status_dev = nullptr;   // one word per slot
    int *status_host = nullptr;  // pinned copies

    std::mutex mu;
    std::condition_variable cv_dispatch, cv_complete, cv_done;
    std::deque<Req *> pending;
    std::deque<Batch *> inflight;
    std::vector<int> free_slots;
    std::unordered_map<long long, Req *> reqs;
    size_t used = 0, peak = 0;
    long long next_id = 0, submitted = 0, completed = 0, failed = 0, batches = 0, batched = 0;
    std::vector<double> lat;
    double flops = 0.0, t_first = -1.0, t_last = 0.0;
    bool stop = false;
    std::thread dispatcher, completer;
};

namespace {

double now_us()
{
    return std::chrono::duration<double, std::micro>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// Device bytes a request may need: its activations and result (host requests),
// between-stage buffers and its share of the grouped tables.
size_t request_bytes(const fg_request &r, int algo)
{
    const int n = r.num_gemm;
    std::vector<long> M(n), K(n);
    size_t tab = 2048;
    for (int i = 0; i < n; ++i) {
        M[i] = r.W[i]->M;
        K[i] = r.W[i]->K;
        const long tiles = ((M[i] + 127) / 128) * ((r.N + 127) / 128);
        tab += 1024 + (size_t)tiles * sizeof(WorkEntry) + (size_t)((r.N + 127) / 128) * 4;
    }
    const int elt = elt_of(r.dtype);
    const int oelt = 4;
    size_t b = group_chain_bytes(r.dtype, algo, r.N, n, M.data(), K.data()) + tab;
    if (r.where == FG_MEM_HOST)
        b += carve_size((size_t)K[0] * r.N * elt) + carve_size((size_t)M[n - 1] * r.N * oelt);
    return b;
}

void server_finish(fg_server_s *s, fg_server_s::Batch *b, double t)
{
    // called with s->mu held
    for (auto *q : b->reqs) {
        q->done = true;
        q->status = b->status;
        q->latency_us = t - q->t_submit;
        if (b->status == FG_OK) {
            s->lat.push_back(q->latency_us);
            s->flops += q->flops;
            ++s->completed;
        } else {
            ++s->failed;
        }
    }
    s->t_last = t;
    s->used -= b->bytes;
    s->free_slots.push_back(b->slot);
}

// Launches one batch on its slot's stream: device copies of host operands,
// one grouped launch per dtype present, copies of host results, an event.
int server_launch(fg_server_s *s, fg_server_s::Batch *b)
{
    DevCtx *c = s->c;
    const int slot = b->slot;
    cudaStream_t st = s->streams[slot];
    int *status = s->status_dev + slot;
    const int algo = f32_algo();
    const int sem = semantics();
    CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), st));
    CUDA_TRY(cudaMallocFromPoolAsync(&b->mem, b->bytes, s->pool, st));
    Carver cv;
    cv.base = (char *)b->mem;
    // device operands of every request
    std::vector<const void *> dB(b->reqs.size());
    std::vector<void *> dC(b->reqs.size());
    for (size_t i = 0; i < b->reqs.size(); ++i) {
        const fg_request &r = b->reqs[i]->r;
        const int n = r.num_gemm;
        const long K0 = r.W[0]->K, Mn = r.W[n - 1]->M;
        if (r.where == FG_MEM_HOST) {
            const size_t bb = (size_t)K0 * r.N * elt_of(r.dtype);
            void *p = cv.take(bb);
            CUDA_TRY(cudaMemcpyAsync(p, r.B, bb, cudaMemcpyHostToDevice, st));
            dB[i] = p;
            dC[i] = cv.take((size_t)Mn * r.N * 4);
        } else {
            dB[i] = r.B;
            dC[i] = r.C;
        }
    }
    // one grouped launch per dtype
    size_t tab_total = 0;
    std::vector<std::vector<fg_chain_desc>> per(3);
    const int dts[3] = {FG_DT_BF16, FG_DT_INT8, FG_DT_F32};
    for (size_t i = 0; i < b->reqs.size(); ++i) {
        const fg_request &r = b->reqs[i]->r;
        for (int d = 0; d < 3; ++d)
            if (r.dtype == dts[d])
                per[d].push_back(fg_chain_desc{dC[i], dB[i], r.N, r.num_gemm, r.W});
    }
    b->gx.resize(3);
    const int cap = s->o.ctas_per_batch;
    for (int d = 0; d < 3; ++d) {
        if (per[d].empty()) continue;
        const int a = dts[d] == FG_DT_F32 ? algo : 0;
        int kernel = g_group_kernel.load(), order = g_group_order.load();
        group_resolve(c, dts[d], a, (int)per[d].size(), per[d].data(), kernel, order);
        int e = group_build(c, dts[d], a, kernel, order, (int)per[d].size(), per[d].data(), cv,
                            b->gx[d], status, cap);
        if (e) return e;
        tab_total += group_tab_bytes(b->gx[d]);
    }
    if (cv.off > b->bytes) return fail(FG_ERR_NOMEM, "serving: admission estimate too small");
    CUDA_TRY(cudaMallocFromPoolAsync(&b->tab, tab_total, s->pool, st));
    Carver ct;
    ct.base = (char *)b->tab;
    for (int d = 0; d < 3; ++d) {
        if (per[d].empty()) continue;
        group_place(b->gx[d], ct);
        int e = group_upload(b->gx[d], st, false);
        if (e) return e;
        if ((e = group_launch(c, b->gx[d], st, false, status))) return e;
    }
    for (size_t i = 0; i < b->reqs.size(); ++i) {
        const fg_request &r = b->reqs[i]->r;
        if (r.where != FG_MEM_HOST) continue;
        const int n = r.num_gemm;
        long rows = r.W[n - 1]->M;
        // INT8 reference semantics leave rows >= 4 * floor(M / 4) of C untouched
        if (r.dtype == FG_DT_INT8 && sem == FG_SEM_REF) rows = (rows / 4) * 4;
        if (rows > 0)
            CUDA_TRY(cudaMemcpyAsync(r.C, dC[i], (size_t)rows * r.N * 4, cudaMemcpyDeviceToHost, st));
    }
    CUDA_TRY(cudaMemcpyAsync(s->status_host + slot, status, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaFreeAsync(b->tab, st));
    CUDA_TRY(cudaFreeAsync(b->mem, st));
    CUDA_TRY(cudaEventRecord(s->events[slot], st));
    return FG_OK;
}

void server_dispatch_loop(fg_server_s *s)
{
    cudaSetDevice(s->c->dev);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        if (s->stop && s->pending.empty()) break;
        if (s->pending.empty() || s->free_slots.empty()) {
            s->cv_dispatch.wait_for(lk, std::chrono::milliseconds(5));
            continue;
        }
        // busy device: wait for a full batch or the oldest request's window
        if (!s->inflight.empty() && (int)s->pending.size() < s->o.max_batch && !s->stop) {
            const double waited = now_us() - s->pending.front()->t_submit;
            if (waited < s->o.max_wait_us) {
                s->cv_dispatch.wait_for(
                    lk, std::chrono::microseconds((long)(s->o.max_wait_us - waited) + 1));
                continue;
            }
        }
        auto *b = new fg_server_s::Batch;
        while (!s->pending.empty() && (int)b->reqs.size() < s->o.max_batch) {
            fg_server_s::Req *q = s->pending.front();
            if (s->used + b->bytes + q->bytes > (size_t)s->o.hbm_budget) break;
            b->bytes += q->bytes;
            b->reqs.push_back(q);
            s->pending.pop_front();
        }
        if (b->reqs.empty()) {
            delete b;
            if (s->inflight.empty()) {  // cannot fit even alone: fail it
                fg_server_s::Req *q = s->pending.front();
                s->pending.pop_front();
                q->done = true;
                q->status = FG_ERR_NOMEM;
                ++s->failed;
                s->cv_done.notify_all();
            } else {
                s->cv_dispatch.wait_for(lk, std::chrono::milliseconds(5));
            }
            continue;
        }
        b->slot = s->free_slots.back();
        s->free_slots.pop_back();
        s->used += b->bytes;
        s->peak = std::max(s->peak, s->used);
        ++s->batches;
        s->batched += (long long)b->reqs.size();
        lk.unlock();
        int st;
        {
            std::lock_guard<std::mutex> g(s->c->mu);
            st = server_launch(s, b);
        }
        if (st) {  // nothing more runs for this batch: return its memory to the pool
            cudaGetLastError();
            cudaStream_t bs = s->streams[b->slot];
            if (b->tab) cudaFreeAsync(b->tab, bs);
            if (b->mem) cudaFreeAsync(b->mem, bs);
            cudaStreamSynchronize(bs);
            cudaGetLastError();
        }
        lk.lock();
        b->status = st;
        s->inflight.push_back(b);
        s->cv_complete.notify_one();
    }
}

void server_complete_loop(fg_server_s *s)
{
    cudaSetDevice(s->c->dev);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        while (s->inflight.empty() && !(s->stop && s->pending.empty()))
            s->cv_complete.wait_for(lk, std::chrono::milliseconds(5));
        if (s->inflight.empty()) break;
        fg_server_s::Batch *b = s->inflight.front();
        lk.unlock();
        if (b->status == FG_OK) {
            cudaError_t e = cudaEventSynchronize(s->events[b->slot]);
            if (e != cudaSuccess) {
                cudaGetLastError();
                b->status = FG_ERR_CUDA;
            } else if (s->status_host[b->slot]) {
                b->status = FG_ERR_TIMEOUT;
            }
        }
        const double t = now_us();
        lk.lock();
        s->inflight.pop_front();
        server_finish(s, b, t);
        delete b;
        s->cv_dispatch.notify_one();
        s->cv_done.notify_all();
    }
}

}  // namespace

FG_EXPORT int fg_server_create(const fg_server_opts *opts, fg_server *out)
{
    if (!out) return fail(FG_ERR_INVALID, "null server pointer");
    *out = nullptr;
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    fg_server_s *s = new fg_server_s;
    s->c = c;
    if (opts) s->o = *opts;
    if (s->o.max_batch <= 0) s->o.max_batch = 64;
    if (s->o.slots <= 0) s->o.slots = 2;
    if (s->o.slots > 16) s->o.slots = 16;
    if (s->o.max_wait_us <= 0) s->o.max_wait_us = 200;
    if (s->o.ctas_per_batch <= 0) s->o.ctas_per_batch = std::max(2, c->sms / s->o.slots);
    if (s->o.hbm_budget <= 0) {
        size_t fr = 0, tot = 0;
        CUDA_TRY(cudaMemGetInfo(&fr, &tot));
        s->o.hbm_budget = (long long)(0.8 * (double)fr);
    }
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = c->dev;
    CUDA_TRY(cudaMemPoolCreate(&s->pool, &props));
    uint64_t keep = ~0ull;  // keep freed blocks for the next batches
    CUDA_TRY(cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    s->streams.resize(s->o.slots);
    s->events.resize(s->o.slots);
    for (int i = 0; i < s->o.slots; ++i) {
        CUDA_TRY(cudaStreamCreateWithFlags(&s->streams[i], cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&s->events[i], cudaEventDisableTiming));
        s->free_slots.push_back(s->o.slots - 1 - i);
    }
    CUDA_TRY(cudaMalloc(&s->status_dev, s->o.slots * sizeof(int)));
    CUDA_TRY(cudaMallocHost(&s->status_host, s->o.slots * sizeof(int)));
    s->dispatcher = std::thread(server_dispatch_loop, s);
    s->completer = std::thread(server_complete_loop, s);
    *out = s;
    return ok();
}

FG_EXPORT long long fg_server_submit(fg_server s, const fg_request *r)
{
    if (!s || !r) return -fail(FG_ERR_INVALID, "null server or request");
    if (r->dtype != FG_DT_BF16 && r->dtype != FG_DT_INT8 && r->dtype != FG_DT_F32)
        return -fail(FG_ERR_INVALID, "unknown dtype %d", r->dtype);
    if (!r->W || !r->B || !r->C || r->num_gemm < 1 || r->num_gemm > 4096)
        return -fail(FG_ERR_INVALID, "null pointer or bad GEMM count");
    if (r->where != FG_MEM_HOST && r->where != FG_MEM_DEVICE)
        return -fail(FG_ERR_INVALID, "where must be FG_MEM_HOST or FG_MEM_DEVICE");
    const int elt = elt_of(r->dtype);
    if (r->N <= 0 || r->N > (1l << 30) || (r->N * elt) % 16)
        return -fail(FG_ERR_INVALID, "N must be positive with 16-byte rows");
    if (r->where == FG_MEM_DEVICE && (!aligned16(r->B) || !aligned16(r->C)))
        return -fail(FG_ERR_INVALID, "device pointers must be 16-byte aligned");
    for (int i = 0; i < r->num_gemm; ++i) {
        if (!r->W[i] || r->W[i]->dtype != r->dtype || r->W[i]->dev != s->c->dev)
            return -fail(FG_ERR_INVALID, "gemm %d: weights missing, of another dtype or device",
                         i + 1);
        if (i > 0 && r->W[i]->K != r->W[i - 1]->M)
            return -fail(FG_ERR_INVALID, "gemm %d: K must equal the previous M", i + 1);
        if (r->W[i]->K % 2) return -fail(FG_ERR_INVALID, "gemm %d: K must be even", i + 1);
    }
    auto *q = new fg_server_s::Req;
    q->r = *r;
    q->W.assign(r->W, r->W + r->num_gemm);
    q->r.W = q->W.data();
    q->bytes = request_bytes(q->r, f32_algo());
    for (int i = 0; i < r->num_gemm; ++i) q->flops += gemm_flops(r->W[i]->M, r->N, r->W[i]->K);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
        delete q;
        return -fail(FG_ERR_INVALID, "server is stopping");
    }
    q->id = s->next_id++;
    q->t_submit = now_us();
    if (s->t_first < 0) s->t_first = q->t_submit;
    s->reqs[q->id] = q;
    s->pending.push_back(q);
    ++s->submitted;
    s->cv_dispatch.notify_one();
    ok();
    return q->id;
}

FG_EXPORT int fg_server_wait(fg_server s, long long id, double *latency_us)
{
    if (!s) return fail(FG_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail(FG_ERR_INVALID, "unknown request id %lld", id);
    fg_server_s::Req *q = it->second;
    while (!q->done) s->cv_done.wait(lk);
    const int st = q->status;
    if (latency_us) *latency_us = q->latency_us;
    s->reqs.erase(it);
    delete q;
    if (st) return fail(st, "request %lld failed (status %d)", id, st);
    return ok();
}

FG_EXPORT int fg_server_replay(fg_server s, const fg_request *reqs, int n, const double *at_us,
                               long long *ids)
{
    if (!s || (n > 0 && (!reqs || !at_us || !ids))) return fail(FG_ERR_INVALID, "null pointer");
    const double t0 = now_us();
    for (int i = 0; i < n; ++i) {
        const double due = t0 + at_us[i];
        double t = now_us();
        if (due - t > 300.0)
            std::this_thread::sleep_for(std::chrono::microseconds((long)(due - t - 200.0)));
        while (now_us() < due) {
        }
        ids[i] = fg_server_submit(s, reqs + i);
    }
    return ok();
}

FG_EXPORT int fg_server_drain(fg_server s)
{
    if (!s) return fail(FG_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    while (s->completed + s->failed < s->submitted) s->cv_done.wait(lk);
    return ok();
}

FG_EXPORT int fg_server_get_stats(fg_server s, fg_server_stats *out)
{
    if (!s || !out) return fail(FG_ERR_INVALID, "null pointer");
    std::lock_guard<std::mutex> lk(s->mu);
    memset(out, 0, sizeof *out);
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->failed = s->failed;
    out->batches = s->batches;
    out->mean_batch = s->batches ? (double)s->batched / (double)s->batches : 0.0;
    std::vector<double> v = s->lat;
    if (!v.empty()) {
        std::sort(v.begin(), v.end());
        auto pct = [&](double p) {
            const double x = p * (double)(v.size() - 1);
            const size_t i = (size_t)x;
            const double f = x - (double)i;
            return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
        };
        out->p50_us = pct(0.50);
        out->p99_us = pct(0.99);
        double sum = 0.0;
        for (double x : v) sum += x;
        out->mean_us = sum / (double)v.size();
        out->max_us = v.back();
    }
    out->flops = s->flops;
    out->span_s = s->t_first >= 0 ? (s->t_last - s->t_first) * 1e-6 : 0.0;
    out->peak_bytes = (long long)s->peak;
    return ok();
}

FG_EXPORT int fg_server_reset_stats(fg_server s)
{
    if (!s) return fail(FG_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    s->lat.clear();
    s->submitted -= s->completed + s->failed;
    s->completed = s->failed = 0;
    s->batches = s->batched = 0;
    s->flops = 0.0;
    s->t_first = -1.0;
    s->t_last = 0.0;
    s->peak = s->used;
    return ok();
}

FG_EXPORT int fg_server_destroy(fg_server s)
{
    if (!s) return ok();
    fg_server_drain(s);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_dispatch.notify_all();
    s->cv_complete.notify_all();
    s->dispatcher.join();
    s->completer.join();
    for (auto &kv : s->reqs) delete kv.second;
    for (auto st : s->streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    for (auto e : s->events) cudaEventDestroy(e);
    cudaFree(s->status_dev);
    cudaFreeHost(s->status_host);
    cudaMemPoolDestroy(s->pool);
    delete s;
    return ok();
}
