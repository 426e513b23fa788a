// C ABI of flashgemm-b200: the reference's entry points (flashgemm.h,
// libshalom.h), single chains and SGEMMs on host or device memory, the weight
// registry and per-launch profiling (flashgemm_b200.h), over the CUDA kernels.
// Grouped launches, plans and the autotuner are in fg_group_api.cu, the
// serving loop in fg_serve.cu.
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

#include "fg_host.h"


namespace fg {
namespace host {

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

// INT8 chains' intermediates in L2. By default they are stored with an L2
// evict-last policy: the stage that later overwrites the same ping-pong buffer
// finds the dead lines still in L2, so they are not written back (measured on
// B200, INT8 chain 8192 x 2048 -> 4096 -> 2048 -> 4096 -> 1024: 82 MB of DRAM
// traffic per launch against 97 MB, same kernel time). FG_L2_KEEP=0 stores them
// like any data; a number of MB also sets aside that much of L2 for such lines
// in this process's context (clamped to the device's maximum, 79 MB on B200;
// 62 MB per launch, kernel 1.7 % slower).
struct L2Keep {
    bool hint = true;
    long setaside_mb = 0;
};
const L2Keep &l2_keep()
{
    static const L2Keep k = [] {
        L2Keep r;
        const char *v = getenv("FG_L2_KEEP");
        if (!v || !v[0]) return r;
        if (v[0] == '0' && !v[1]) {
            r.hint = false;
            return r;
        }
        r.setaside_mb = atol(v) > 0 ? atol(v) : 0;
        return r;
    }();
    return k;
}

// ---------------------------------------------------------------- per-device context


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
        c->work = c->stream;
        CUDA_TRY(cudaEventCreateWithFlags(&c->ev_in, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&c->ev_out, cudaEventDisableTiming));
        CUDA_TRY(cudaStreamCreateWithFlags(&c->stream_h2d, cudaStreamNonBlocking));
        CUDA_TRY(cudaStreamCreateWithFlags(&c->stream_d2h, cudaStreamNonBlocking));
        for (int j = 0; j < DevCtx::kCopyChunks; ++j) {
            CUDA_TRY(cudaEventCreateWithFlags(&c->ev_up[j], cudaEventDisableTiming));
            CUDA_TRY(cudaEventCreateWithFlags(&c->ev_done[j], cudaEventDisableTiming));
            CUDA_TRY(cudaEventCreateWithFlags(&c->ev_down[j], cudaEventDisableTiming));
        }
        CUDA_TRY(cudaMalloc(&c->status, sizeof(int)));
        CUDA_TRY(cudaMemset(c->status, 0, sizeof(int)));
        CUDA_TRY(cudaMallocHost(&c->status_host, sizeof(int)));
        if (l2_keep().setaside_mb > 0) {  // a tuning: where the device refuses it, run without
            int mx = 0;
            const size_t want = (size_t)l2_keep().setaside_mb << 20;
            if (cudaDeviceGetAttribute(&mx, cudaDevAttrMaxPersistingL2CacheSize, dev) != cudaSuccess ||
                cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize,
                                   want < (size_t)mx ? want : (size_t)mx) != cudaSuccess)
                cudaGetLastError();
        }
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
    CUDA_TRY(cudaStreamSynchronize(c->work));
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
    CUDA_TRY(cudaStreamSynchronize(c->work));
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

int enter_stream(DevCtx *c, cudaStream_t s)
{
    if (s == c->work) return FG_OK;
    CUDA_TRY(cudaEventRecord(c->ev_in, c->work));
    CUDA_TRY(cudaStreamWaitEvent(s, c->ev_in, 0));
    c->work = s;
    return FG_OK;
}

// Counters are carved in 64-int steps from a block of 1 Mi ints (grown when a
// launch needs more); a used-up block is zeroed by one memset on the work
// stream, which every earlier launch precedes, so no launch sees another's counts.
int take_counters(DevCtx *c, size_t n, int **out)
{
    const size_t need = (n + 63) & ~(size_t)63;
    if (need > c->ctr_cap) {
        CUDA_TRY(cudaStreamSynchronize(c->work));
        if (c->ctr) cudaFree(c->ctr);
        c->ctr = nullptr;
        c->ctr_cap = 0;
        const size_t cap = need > (1u << 20) ? need : (1u << 20);
        cudaError_t e = cudaMalloc(&c->ctr, cap * sizeof(int));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(FG_ERR_NOMEM, "chain counters: %s", cudaGetErrorString(e));
        }
        CUDA_TRY(cudaMemsetAsync(c->ctr, 0, cap * sizeof(int), c->work));
        c->ctr_cap = cap;
        c->ctr_off = 0;
    } else if (c->ctr_off + need > c->ctr_cap) {
        CUDA_TRY(cudaMemsetAsync(c->ctr, 0, c->ctr_cap * sizeof(int), c->work));
        c->ctr_off = 0;
    }
    *out = c->ctr + c->ctr_off;
    c->ctr_off += need;
    return FG_OK;
}



// ---------------------------------------------------------------- chain core



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
        s += carve_size(chain_counter_ints(n, M, N) * sizeof(int));
        if (getenv("FG_TRACE_DIR")) {  // per-tile timeline of the fused kernel
            size_t items = 0;
            for (int i = 0; i < n; ++i) items += (size_t)((M[i] + 255) / 256) * ((N + 255) / 256);
            s += carve_size(items * 2 * 10 * 8);
            // or of the narrow kernel: one row per (column block, unit) at most
            s += carve_size((size_t)((N + 127) / 128) * (n - 1 + (M[n - 1] + 127) / 128) *
                            kNarrowTraceFields * 8);
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
        if (getenv("FG_TRACE_DIR"))  // per-tile timeline of the panel-resident kernel
            s += carve_size((size_t)((N + 127) / 128) * kPanelMaxStages * kPanelTraceFields * 8);
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

// Chains whose intermediates fit on chip: FG_NARROW_AUTO (default), _ALWAYS
// or _OFF; the environment variable FG_NARROW (0 / 1) sets the initial mode.
std::atomic<int> g_narrow_mode{-1};
int narrow_mode()
{
    int m = g_narrow_mode.load();
    if (m < 0) {
        const char *v = getenv("FG_NARROW");
        m = v && v[0] == '0' ? FG_NARROW_OFF : v && v[0] == '1' ? FG_NARROW_ALWAYS : FG_NARROW_AUTO;
        g_narrow_mode.store(m);
    }
    return m;
}

int launch_stages(DevCtx *c, int kind, std::vector<StageArgs> &stages, long N)
{
    const int n = (int)stages.size();
    const int nm = fused_enabled() ? narrow_mode() : FG_NARROW_OFF;
    if (nm != FG_NARROW_OFF && narrow_eligible(stages.data(), n) &&
        (nm == FG_NARROW_ALWAYS || narrow_preferred(stages.data(), n, c->sms))) {
        // intermediates on chip; a chain whose operands the tensor maps cannot
        // describe (unaligned rows) falls through to the fused chain
        static thread_local NarrowArgs P;
        int grid = 0;
        if (plan_narrow(stages.data(), n, c->sms, P, grid) == cudaSuccess) {
            double fl = 0.0;
            for (auto &st : stages) fl += gemm_flops(st.M, st.N, st.K);
            // FG_TRACE_DIR=<dir>: a per-unit timeline of every narrow launch
            static const char *trace_dir = getenv("FG_TRACE_DIR");
            size_t trace_words = 0;
            P.trace = nullptr;
            if (trace_dir) {
                P.trace_units = narrow_units_per_cta(P, grid);
                trace_words = (size_t)grid * P.trace_units * kNarrowTraceFields;
                P.trace = (unsigned long long *)arena_take(c, trace_words * 8);
                CUDA_TRY(cudaMemsetAsync(P.trace, 0, trace_words * 8, c->work));
            }
            const int st = run_kernel(c, kind, fl, "narrow chain",
                                      [&] { return launch_narrow(P, grid, c->status, c->work); });
            if (st == FG_OK && P.trace) {
                std::vector<unsigned long long> h(trace_words);
                CUDA_TRY(cudaMemcpyAsync(h.data(), P.trace, trace_words * 8,
                                         cudaMemcpyDeviceToHost, c->work));
                CUDA_TRY(cudaStreamSynchronize(c->work));
                static int seq = 0;
                char path[1024];
                snprintf(path, sizeof path, "%s/narrow_trace_%d.csv", trace_dir, seq++);
                if (FILE *f = fopen(path, "w")) {
                    fprintf(f, "cta,unit,stage,pos,row0,tiles,sm,prod_start,prod_end,mma_wait,"
                               "mma_start,mma_end,epi_start,epi_end\n");
                    for (size_t r = 0; r < trace_words / kNarrowTraceFields; ++r) {
                        const unsigned long long *v = &h[r * kNarrowTraceFields];
                        if (!v[1]) continue;  // a unit the CTA did not have
                        fprintf(f, "%zu,%zu,%llu,%llu,%llu,%llu,%llu", r / P.trace_units,
                                r % P.trace_units, v[0] & 0xff, (v[0] >> 8) & 0xffff,
                                (v[0] >> 24) & 0xff, (v[0] >> 32) & 0xff, v[0] >> 40);
                        for (int k = 1; k < kNarrowTraceFields; ++k) fprintf(f, ",%llu", v[k]);
                        fprintf(f, "\n");
                    }
                    fclose(f);
                }
            }
            P.trace = nullptr;
            return st;
        }
        cudaGetLastError();
    }
    if (fused_enabled() && n <= chain_max_stages() && !g_fused_unsupported[c->dev & 63]) {
        const long tiles_n = (N + 255) / 256;
        std::vector<long> rows(n);
        for (int i = 0; i < n; ++i) rows[i] = stages[i].M;
        const size_t done_ints = chain_counter_ints(n, rows.data(), N);
        int *done = nullptr;
        if (int e = take_counters(c, done_ints, &done)) return e;
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
            CUDA_TRY(cudaMemsetAsync(trace, 0, trace_words * 8, c->work));
        }
        cudaError_t le = cudaSuccess;
        int st = run_kernel(c, kind, fl, "fused chain", [&] {
            le = launch_tc_chain(stages.data(), n, done, c->status, trace, c->sms, c->work);
            return le;
        });
        if (st == FG_OK && trace) {
            std::vector<unsigned long long> h(trace_words);
            CUDA_TRY(cudaMemcpyAsync(h.data(), trace, trace_words * 8, cudaMemcpyDeviceToHost,
                                     c->work));
            CUDA_TRY(cudaStreamSynchronize(c->work));
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
                            [&] { return launch_tc_stage(s, c->sms, c->work); });
        if (st) return st;
    }
    return FG_OK;
}


// Builds the stage list of a BF16 or INT8 chain (between-stage buffers from the
// arena, weight preparations launched on c->work) without launching the stages.
int build_tc_stages(DevCtx *c, int dtype, int sem, void *C, long ldc, Mat b, long N, int n,
                    const Mat *a, const long *M, const long *K, const PreparedW *pw,
                    std::vector<StageArgs> &out, Carver *cv)
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
                CUDA_TRY(cudaMemsetAsync(wp, 0, (size_t)M[i] * ldk * 2, c->work));
                CUDA_TRY(cudaMemcpy2DAsync(wp, ldk * 2, w, ldw * 2, K[i] * 2, M[i],
                                           cudaMemcpyDeviceToDevice, c->work));
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
                // a padded copy: a job of the same batched launch as the tail blocks
                uint8_t *wp = (uint8_t *)take((size_t)Mi * ldw);
                if (jobs.n == 8) {  // flush a full batch
                    int st = run_kernel(c, FG_PK_AUX, 0.0, "int8 weight prep",
                                        [&] { return launch_prep_int8_jobs(jobs, c->work); });
                    if (st) return st;
                    jobs.n = 0;
                }
                jobs.job[jobs.n++] = PrepJob{(const int8_t *)a[i].p, a[i].ld, wp, ldw, Mi, Ki, 0, 0};
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
                    int st = run_kernel(c, FG_PK_AUX, 0.0, "int8 weight prep",
                                        [&] { return launch_prep_int8_jobs(jobs, c->work); });
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
            s.l2_keep = (!last && l2_keep().hint) ? 1 : 0;
            s.m_written = (last && ref) ? (int)((Mi / 4) * 4) : (int)Mi;
            s.tail_lo = (int)tail_lo;
            s.tail_hi = (int)tail_hi;
            stages.push_back(s);
            x = s.out;
            ldx = s.ld_out;
        }
        if (jobs.n) {  // the chain's padded copies and tail blocks in one launch
            int st = run_kernel(c, FG_PK_AUX, 0.0, "int8 weight prep",
                                [&] { return launch_prep_int8_jobs(jobs, c->work); });
            if (st) return st;
        }
        out = std::move(stages);
        return FG_OK;
    }
    return fail(FG_ERR_INVALID, "not a tensor-core chain dtype");
}

// Runs the chain on c->work. Device operands: B (K[0] x N, ld b.ld),
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
                                [&] { return launch_ffma_sgemm(f, c->sms, c->work); });
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
                                         c->work);
            });
            if (st) return st;
        }
        if (fused_enabled() && panel_enabled() && panel_eligible(N, n, M, K) &&
            aligned16(b.p) && aligned16(C) && b.ld % 4 == 0 && ldc % 4 == 0) {
            // every dimension fits on chip: one launch, intermediates in shared memory
            PanelChainArgs pa;
            memset(&pa, 0, sizeof pa);
            pa.n = n;
            pa.N = N;
            pa.B = (const float *)b.p;
            pa.ldb = b.ld;
            pa.C = (float *)C;
            pa.ldc = ldc;
            for (int i = 0; i < n; ++i) {
                pa.w_hi[i] = wh[i];
                pa.w_lo[i] = wl[i];
                pa.ldw[i] = wld[i];
                pa.M[i] = M[i];
                pa.K[i] = K[i];
                pa.kchunk[i] = tf32_chunk_blocks(K[i]);
            }
            double fl = 0.0;
            for (int i = 0; i < n; ++i) fl += gemm_flops(M[i], N, K[i]);
            const long nblocks = (N + 127) / 128;
            // FG_TRACE_DIR=<dir>: a per-tile timeline of every panel launch
            static const char *trace_dir = getenv("FG_TRACE_DIR");
            const size_t trace_words = (size_t)nblocks * kPanelMaxStages * kPanelTraceFields;
            unsigned long long *trace = nullptr;
            if (trace_dir) {
                trace = (unsigned long long *)arena_take(c, trace_words * 8);
                CUDA_TRY(cudaMemsetAsync(trace, 0, trace_words * 8, c->work));
            }
            int st = run_kernel(c, FG_PK_TC_TF32X3, fl, "panel-resident chain", [&] {
                return launch_panel_one(pa, c->sms, c->status, c->work, trace);
            });
            if (st == FG_OK && trace) {
                std::vector<unsigned long long> h(trace_words);
                CUDA_TRY(cudaMemcpyAsync(h.data(), trace, trace_words * 8, cudaMemcpyDeviceToHost,
                                         c->work));
                CUDA_TRY(cudaStreamSynchronize(c->work));
                static int seq = 0;
                char path[1024];
                snprintf(path, sizeof path, "%s/panel_trace_%d.csv", trace_dir, seq++);
                if (FILE *f = fopen(path, "w")) {
                    fprintf(f, "pos,stage,slot,sm,cta,prod_start,prod_end,mma_wait,mma_start,mma_end,"
                               "epi_start,epi_end,split_start,split_end\n");
                    for (size_t r = 0; r < trace_words / kPanelTraceFields; ++r) {
                        const unsigned long long *v = &h[r * kPanelTraceFields];
                        if (!v[1]) continue;  // no such tile
                        fprintf(f, "%zu,%zu,%llu,%llu,%llu", r / kPanelMaxStages, r % kPanelMaxStages,
                                v[0] & 0xff, (v[0] >> 16) & 0xffff, v[0] >> 32);
                        for (int k = 1; k < kPanelTraceFields; ++k) fprintf(f, ",%llu", v[k]);
                        fprintf(f, "\n");
                    }
                    fclose(f);
                }
            }
            return st;
        }
        float *xh = (float *)arena_take(c, (size_t)K[0] * ldN * 4);
        float *xl = (float *)arena_take(c, (size_t)K[0] * ldN * 4);
        int st = run_kernel(c, FG_PK_AUX, 0.0, "tf32 split (activations)", [&] {
            return launch_split_tf32((const float *)b.p, b.ld, xh, xl, ldN, K[0], N, c->work);
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
                            [&] { return launch_tc_stage(s, c->sms, c->work); });
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

// Read and clear the device status word (waits for the work stream).
int collect_status(DevCtx *c)
{
    CUDA_TRY(cudaMemcpyAsync(c->status_host, c->status, sizeof(int), cudaMemcpyDeviceToHost,
                             c->work));
    CUDA_TRY(cudaStreamSynchronize(c->work));
    const int code = *c->status_host;
    if (code) {
        CUDA_TRY(cudaMemsetAsync(c->status, 0, sizeof(int), c->work));
        CUDA_TRY(cudaStreamSynchronize(c->work));
        return fail(FG_ERR_TIMEOUT, "a kernel's pipeline wait ran out (code 0x%x)", code);
    }
    return FG_OK;
}

// A pitched copy, issued as one linear copy when both sides are contiguous rows.
// (Measured on B200 with pinned host memory: pitched copies of 512 B to 16 KB
// rows move at the linear rate, about 55 GB/s each way, so either form serves.)
cudaError_t copy_rows(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width,
                      size_t height, cudaMemcpyKind kind, cudaStream_t s)
{
    if (dpitch == width && spitch == width) return cudaMemcpyAsync(dst, src, width * height, kind, s);
    return cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, kind, s);
}

// ---------------------------------------------------------------- host copies

RowCopier::RowCopier(int threads) : parts_(threads < 1 ? 1 : threads)
{
    for (int i = 1; i < parts_; ++i) th_.emplace_back([this, i] { run(i); });
}

RowCopier::~RowCopier()
{
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_.store(true);
    }
    cv_go_.notify_all();
    for (auto &t : th_) t.join();
}

namespace {
void copy_part(char *dst, size_t dpitch, const char *src, size_t spitch, size_t width, size_t r0,
               size_t r1)
{
    if (r1 <= r0) return;
    if (dpitch == width && spitch == width) {
        memcpy(dst + r0 * width, src + r0 * width, (r1 - r0) * width);
        return;
    }
    for (size_t r = r0; r < r1; ++r) memcpy(dst + r * dpitch, src + r * spitch, width);
}

// Spin this long for the next piece before sleeping: the pieces of one call
// follow each other within microseconds, and a sleeping worker's wake-up costs
// tens of microseconds.
constexpr int kSpinUs = 200;
}  // namespace

void RowCopier::run(int part)
{
    unsigned long long seen = 0;
    while (true) {
        const auto t0 = std::chrono::steady_clock::now();
        while (gen_.load(std::memory_order_acquire) == seen && !stop_.load()) {
            if (std::chrono::steady_clock::now() - t0 > std::chrono::microseconds(kSpinUs)) {
                std::unique_lock<std::mutex> lk(mu_);
                cv_go_.wait(lk, [&] { return stop_.load() || gen_.load() != seen; });
                break;
            }
        }
        if (stop_.load()) return;
        seen = gen_.load(std::memory_order_acquire);
        copy_part(dst_, dpitch_, src_, spitch_, width_, height_ * part / parts_,
                  height_ * (part + 1) / parts_);
        if (pending_.fetch_sub(1, std::memory_order_acq_rel) == 1) {
            std::lock_guard<std::mutex> lk(mu_);
            cv_done_.notify_one();
        }
    }
}

void RowCopier::copy(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width,
                     size_t height)
{
    char *d = static_cast<char *>(dst);
    const char *sp = static_cast<const char *>(src);
    if (parts_ == 1 || height < (size_t)parts_ || width * height < (256u << 10)) {
        copy_part(d, dpitch, sp, spitch, width, 0, height);
        return;
    }
    // the job's fields are published by the release increment of gen_
    dst_ = d;
    src_ = sp;
    dpitch_ = dpitch;
    spitch_ = spitch;
    width_ = width;
    height_ = height;
    pending_.store(parts_ - 1, std::memory_order_relaxed);
    {
        std::lock_guard<std::mutex> lk(mu_);  // a worker about to sleep sees the new generation
        gen_.fetch_add(1, std::memory_order_release);
    }
    cv_go_.notify_all();
    copy_part(d, dpitch, sp, spitch, width, 0, height / parts_);
    const auto t0 = std::chrono::steady_clock::now();
    while (pending_.load(std::memory_order_acquire) != 0) {
        if (std::chrono::steady_clock::now() - t0 > std::chrono::microseconds(kSpinUs)) {
            std::unique_lock<std::mutex> lk(mu_);
            cv_done_.wait(lk, [&] { return pending_.load() == 0; });
            break;
        }
    }
}

// How a host operand reaches the device: page-locked memory (or managed) is
// copied by DMA directly; ordinary pageable memory goes through pinned staging.
enum class HostMem { Pinned, Pageable, Device };
HostMem host_mem(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return HostMem::Pageable;
    }
    if (a.type == cudaMemoryTypeDevice) return HostMem::Device;
    return a.type == cudaMemoryTypeUnregistered ? HostMem::Pageable : HostMem::Pinned;
}

int pin_reserve(DevCtx *c, size_t bytes)
{
    if (bytes <= c->pin_cap) return FG_OK;
    if (c->pin) cudaFreeHost(c->pin);  // every earlier host-pointer call has completed
    c->pin = nullptr;
    c->pin_cap = 0;
    const size_t cap = bytes + bytes / 4;
    cudaError_t e = cudaMallocHost(&c->pin, cap);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(FG_ERR_NOMEM, "pinned staging of %zu bytes: %s", cap, cudaGetErrorString(e));
    }
    c->pin_cap = cap;
    if (!c->copier) {
        // FG_COPY_THREADS overrides the count (default: half the host's threads, at most 8)
        const char *v = getenv("FG_COPY_THREADS");
        const unsigned hw = std::thread::hardware_concurrency();
        const int n = v ? atoi(v) : (int)std::max(1u, std::min(8u, hw / 2));
        c->copier.reset(new RowCopier(std::max(1, std::min(64, n))));
    }
    return FG_OK;
}

// Host-pointer chain: stage operands into device scratch, run, copy C back.
// B and C rows are ldb and ldc elements apart (N for the reference's dense
// operands; a column slice of a wider chain otherwise).
//
// Column chunks (fused BF16 / INT8 chains from 1024 columns): the weights and
// then each chunk of B go up on one copy stream, each chunk's chain runs on the
// compute stream once its columns are there, and its columns of C come back on
// a second copy stream while later chunks compute. Chunks start on multiples
// of 256 columns: every tile, panel and result is the one of the whole chain.
// Operands in ordinary (pageable) host memory, which the reference's callers
// pass (posix_memalign / malloc), pass through pinned staging: the copier's
// threads move each piece while the copy engines move the previous one, the
// weights in pieces of about 2 MB, B and C chunk by chunk, so that the overlap
// survives; page-locked operands are copied directly.
int host_chain(int dtype, void *C, const void *B, long N, int n, const void *const *A,
               const long *M, const long *K, long ldb, long ldc)
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
    // INT8 reference semantics leave rows >= 4 * floor(M / 4) of C untouched
    // (multigemm/src/kernel_int8.h:943-945)
    long rows = M[n - 1];
    if (dtype == FG_DT_INT8 && sem == FG_SEM_REF) rows = (rows / 4) * 4;

    // which operands need staging, and the pinned bytes they take
    const HostMem mb = host_mem(B), mc = host_mem(C);
    std::vector<HostMem> ma(n);
    for (int i = 0; i < n; ++i) ma[i] = host_mem(A[i]);
    bool dev_ptr = mb == HostMem::Device || mc == HostMem::Device;
    for (int i = 0; i < n; ++i) dev_ptr = dev_ptr || ma[i] == HostMem::Device;
    if (dev_ptr)
        return fail(FG_ERR_INVALID, "host pointers expected (use fg_chain_dev for device memory)");
    size_t pin_bytes = 0;
    std::vector<size_t> pin_w(n, 0);
    for (int i = 0; i < n; ++i)
        if (ma[i] == HostMem::Pageable) {
            pin_w[i] = pin_bytes;
            pin_bytes += carve_size((size_t)M[i] * K[i] * elt);
        }
    const size_t pin_b = pin_bytes;
    if (mb == HostMem::Pageable) pin_bytes += carve_size((size_t)K[0] * N * elt) + 256 * 4;
    const size_t pin_c = pin_bytes;
    if (mc == HostMem::Pageable) pin_bytes += carve_size((size_t)rows * N * out_elt) + 256 * 4;
    if (pin_bytes && (st = pin_reserve(c, pin_bytes))) return st;

    if ((st = enter_stream(c, c->stream))) return st;
    if ((st = arena_reserve(c, need))) return st;
    // the uploads overwrite the arena: after every earlier call's kernels
    CUDA_TRY(cudaEventRecord(c->ev_in, c->stream));
    CUDA_TRY(cudaStreamWaitEvent(c->stream_h2d, c->ev_in, 0));

    void *bd = arena_take(c, (size_t)K[0] * ldN * elt);
    std::vector<Mat> ad(n);
    std::vector<void *> wd(n);
    for (int i = 0; i < n; ++i) {
        wd[i] = arena_take(c, (size_t)M[i] * lda[i] * elt);
        ad[i] = Mat{wd[i], lda[i]};
    }
    void *cd = arena_take(c, (size_t)M[n - 1] * ldN * out_elt);

    const bool chunked = (dtype == FG_DT_BF16 || dtype == FG_DT_INT8) && fused_enabled() &&
                         N >= 1024;
    const int nchunk = chunked ? DevCtx::kCopyChunks : 1;
    const long cw = chunked ? round_up((N + nchunk - 1) / nchunk, 256) : N;
    auto drain = [&] {  // no copy may still touch the caller's buffers after a failure
        cudaStreamSynchronize(c->stream_h2d);
        cudaStreamSynchronize(c->stream);
        cudaStreamSynchronize(c->stream_d2h);
    };
    for (int i = 0; i < n; ++i) {
        cudaError_t e = cudaSuccess;
        const size_t row = (size_t)K[i] * elt;
        if (ma[i] == HostMem::Pageable) {
            // in pieces of about 2 MB: the next piece is staged while this one moves
            char *pw = c->pin + pin_w[i];
            const long piece = std::max(1l, (long)((2u << 20) / std::max<size_t>(row, 1)));
            for (long r0 = 0; r0 < M[i] && e == cudaSuccess; r0 += piece) {
                const long r1 = std::min(M[i], r0 + piece);
                c->copier->copy(pw + r0 * row, row, static_cast<const char *>(A[i]) + r0 * row, row,
                                row, r1 - r0);
                e = copy_rows(static_cast<char *>(wd[i]) + r0 * lda[i] * elt, lda[i] * elt,
                              pw + r0 * row, row, row, r1 - r0, cudaMemcpyHostToDevice,
                              c->stream_h2d);
            }
        } else {
            e = copy_rows(wd[i], lda[i] * elt, A[i], row, row, M[i], cudaMemcpyHostToDevice,
                          c->stream_h2d);
        }
        if (e != cudaSuccess) {
            drain();
            return fail(FG_ERR_CUDA, "chain upload: %s", cudaGetErrorString(e));
        }
    }
    const size_t mark = c->arena_off;
    int chunks = 0;
    // pageable C: each chunk leaves staging once its download has landed,
    // between the later chunks' staging (opportunistically) or at the end
    int copied_out = 0;
    auto copy_out = [&](int jo) {
        const long o0 = jo * cw, o1 = o0 + cw < N ? o0 + cw : N;
        const size_t wo = (size_t)(o1 - o0) * out_elt;
        c->copier->copy(static_cast<char *>(C) + o0 * out_elt, ldc * out_elt,
                        c->pin + pin_c + (size_t)rows * o0 * out_elt, wo, wo, rows);
    };
    for (int j = 0; j < nchunk; ++j) {
        const long c0 = j * cw, c1 = c0 + cw < N ? c0 + cw : N;
        if (c0 >= N) break;
        ++chunks;
        if (mc == HostMem::Pageable && rows > 0)
            while (copied_out < j && cudaEventQuery(c->ev_down[copied_out]) == cudaSuccess)
                copy_out(copied_out++);
        const size_t wb = (size_t)(c1 - c0) * elt;
        char *bj = static_cast<char *>(bd) + c0 * elt;
        char *cj = static_cast<char *>(cd) + c0 * out_elt;
        cudaError_t e;
        if (mb == HostMem::Pageable) {
            char *pb = c->pin + pin_b + (size_t)K[0] * c0 * elt;  // chunk j's columns, dense
            c->copier->copy(pb, wb, static_cast<const char *>(B) + c0 * elt, ldb * elt, wb, K[0]);
            e = copy_rows(bj, ldN * elt, pb, wb, wb, K[0], cudaMemcpyHostToDevice, c->stream_h2d);
        } else {
            e = copy_rows(bj, ldN * elt, static_cast<const char *>(B) + c0 * elt, ldb * elt, wb,
                          K[0], cudaMemcpyHostToDevice, c->stream_h2d);
        }
        if (e == cudaSuccess) e = cudaEventRecord(c->ev_up[j], c->stream_h2d);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, c->ev_up[j], 0);
        if (e != cudaSuccess) {
            drain();
            return fail(FG_ERR_CUDA, "chain upload: %s", cudaGetErrorString(e));
        }
        c->arena_off = mark;  // chunks reuse the scratch in stream order
        if ((st = run_chain(c, dtype, sem, algo, cj, ldN, Mat{bj, ldN}, c1 - c0, n, ad.data(),
                            M, K))) {
            drain();
            return st;
        }
        e = cudaEventRecord(c->ev_done[j], c->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream_d2h, c->ev_done[j], 0);
        const size_t wc = (size_t)(c1 - c0) * out_elt;
        if (e == cudaSuccess && rows > 0) {
            if (mc == HostMem::Pageable)
                e = copy_rows(c->pin + pin_c + (size_t)rows * c0 * out_elt, wc, cj, ldN * out_elt,
                              wc, rows, cudaMemcpyDeviceToHost, c->stream_d2h);
            else
                e = copy_rows(static_cast<char *>(C) + c0 * out_elt, ldc * out_elt, cj,
                              ldN * out_elt, wc, rows, cudaMemcpyDeviceToHost, c->stream_d2h);
        }
        if (e == cudaSuccess) e = cudaEventRecord(c->ev_down[j], c->stream_d2h);
        if (e != cudaSuccess) {
            drain();
            return fail(FG_ERR_CUDA, "chain download: %s", cudaGetErrorString(e));
        }
    }
    if (mc == HostMem::Pageable && rows > 0) {
        // the chunks of C not yet out of staging, each as soon as it has arrived
        for (int j = copied_out; j < chunks; ++j) {
            const cudaError_t e = cudaEventSynchronize(c->ev_down[j]);
            if (e != cudaSuccess) {
                drain();
                return fail(FG_ERR_CUDA, "chain download: %s", cudaGetErrorString(e));
            }
            copy_out(j);
        }
    }
    CUDA_TRY(cudaStreamSynchronize(c->stream_d2h));
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
    return host_chain(dtype, C, B, N, num_gemm, A.data(), M.data(), K.data(), N, N);
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
                          [&] { return launch_ffma_sgemm(f, c->sms, c->work); });
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
    if ((st = enter_stream(c, c->stream))) return st;
    if ((st = arena_reserve(c, need))) return st;
    float *ad = (float *)arena_take(c, (size_t)M * ldk * 4);
    float *bd = (float *)arena_take(c, (size_t)(K > 0 ? K : 1) * ldn * 4);
    float *cd = (float *)arena_take(c, (size_t)M * ldn * 4);
    if (K > 0) {
        CUDA_TRY(copy_rows(ad, ldk * 4, A, K * 4, K * 4, M, cudaMemcpyHostToDevice, c->stream));
        CUDA_TRY(copy_rows(bd, ldn * 4, B, N * 4, N * 4, K, cudaMemcpyHostToDevice, c->stream));
    }
    // singlegemm blocks K by GEMM_K = 2048 and adds the partial sums into C
    // (singlegemm/src/NN_mp.h:13, :247)
    if ((st = run_sgemm(c, algo, cd, ldn, ad, ldk, bd, ldn, M, N, K, 2048))) return st;
    CUDA_TRY(copy_rows(C, N * 4, cd, ldn * 4, N * 4, M, cudaMemcpyDeviceToHost, c->stream));
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

}  // namespace host
}  // namespace fg

// ---------------------------------------------------------------- weight registry


namespace fg {
namespace host {

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
    if ((st = enter_stream(c, c->stream))) return st;
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

}  // namespace host
}  // namespace fg

using namespace fg;
using namespace fg::host;

// Status setters for the library's other host files (fg_noalloc.cu).
namespace fg {
int api_fail(int status, const char *msg) { return host::fail(status, "%s", msg); }
int api_ok() { return host::ok(); }
int noalloc_take_status(int dev, int *code);  // fg_noalloc.cu
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
FG_EXPORT void fg_set_narrow(int mode)
{
    g_narrow_mode.store(mode == FG_NARROW_OFF || mode == FG_NARROW_ALWAYS ? mode : FG_NARROW_AUTO);
}
FG_EXPORT int fg_get_narrow(void) { return narrow_mode(); }
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
    // the kernels run on the caller's stream itself (after all earlier library work)
    if ((st = enter_stream(c, user_stream(stream)))) return st;
    if ((st = arena_reserve(c, need))) return st;
    Mat b{B, N};
    if (pad_b) {
        void *p = arena_take(c, (size_t)K[0] * ldN * elt);
        CUDA_TRY(cudaMemcpy2DAsync(p, ldN * elt, B, N * elt, N * elt, K[0], cudaMemcpyDeviceToDevice,
                                   c->work));
        b = Mat{p, ldN};
    }
    std::vector<Mat> a(num_gemm);
    for (int i = 0; i < num_gemm; ++i) a[i] = Mat{A[i], K[i]};
    if ((st = run_chain(c, dtype, semantics(), algo, C, N, b, N, num_gemm, a.data(), M, K)))
        return st;
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
    if ((st = enter_stream(c, user_stream(stream)))) return st;
    if ((st = arena_reserve(c, need))) return st;
    if ((st = run_sgemm(c, algo, C, N, A, K, B, N, M, N, K, 2048))) return st;
    return ok();
}

FG_EXPORT int fg_sync(void)
{
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    std::lock_guard<std::mutex> lk(c->mu);
    CUDA_TRY(cudaStreamSynchronize(c->work));
    if ((st = collect_status(c))) return st;
    // the allocation-free entry point's own status word (calls made with status == NULL)
    int code = 0;
    const int e = noalloc_take_status(c->dev, &code);
    if (e) return fail(FG_ERR_CUDA, "no-alloc status word: %s", cudaGetErrorString((cudaError_t)e));
    if (code)
        return fail(FG_ERR_TIMEOUT, "fg_chain_bf16_noalloc: a kernel's pipeline wait ran out "
                                    "(code 0x%x)", code);
    return ok();
}

// Columns [c0, c1) of N that part `index` of `parts` owns when one chain is
// split: whole 32-column panels (the reference's between-stage permutation
// never crosses one), as even as the panel count allows, the first parts one
// panel larger.
FG_EXPORT int fg_split_columns(long N, int parts, int index, long *c0, long *c1)
{
    if (N < 0 || parts < 1 || index < 0 || index >= parts || !c0 || !c1)
        return fail(FG_ERR_INVALID, "bad split arguments");
    const long panels = (N + 31) / 32;
    const long per = panels / parts, extra = panels % parts;
    const long p0 = index * per + std::min<long>(index, extra);
    const long p1 = p0 + per + (index < extra ? 1 : 0);
    *c0 = std::min(p0 * 32, N);
    *c1 = std::min(p1 * 32, N);
    return ok();
}

FG_EXPORT int fg_chain_multi_device(int dtype, void *C, const void *B, long N, int num_gemm,
                                    const void *const *A, const long *M, const long *K, int ndev,
                                    const int *devices)
{
    if (dtype != FG_DT_F32 && dtype != FG_DT_BF16 && dtype != FG_DT_INT8)
        return fail(FG_ERR_INVALID, "unknown dtype %d", dtype);
    if (!C || !B || !A || !M || !K || !devices || ndev < 1 || ndev > 64)
        return fail(FG_ERR_INVALID, "null pointer or bad device count");
    int st = check_shapes(dtype, N, num_gemm, M, K);
    if (st) return st;
    for (int i = 0; i < num_gemm; ++i)
        if (K[i] % 2 != 0) return fail(FG_ERR_INVALID, "gemm %d: K must be a multiple of 2", i + 1);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess) {
        cudaGetLastError();
        return fail(FG_ERR_NO_DEVICE, "no CUDA device");
    }
    for (int d = 0; d < ndev; ++d)
        if (devices[d] < 0 || devices[d] >= count)
            return fail(FG_ERR_INVALID, "device %d out of range (%d devices)", devices[d], count);
    const int elt = elt_of(dtype);
    // every part on its own host thread, its device current there; C's slices
    // are disjoint, so the parts share nothing but the caller's read-only inputs
    std::vector<int> status(ndev, FG_OK);
    std::vector<std::string> msg(ndev);
    std::vector<std::thread> th;
    for (int d = 0; d < ndev; ++d) {
        long c0 = 0, c1 = 0;
        fg_split_columns(N, ndev, d, &c0, &c1);
        if (c1 <= c0) continue;
        th.emplace_back([&, d, c0, c1] {
            cudaSetDevice(devices[d]);
            status[d] = host_chain(dtype, static_cast<char *>(C) + c0 * 4,
                                   static_cast<const char *>(B) + c0 * elt, c1 - c0, num_gemm, A, M,
                                   K, N, N);
            if (status[d]) msg[d] = t_msg;
        });
    }
    for (auto &t : th) t.join();
    for (int d = 0; d < ndev; ++d)
        if (status[d]) return fail(status[d], "device %d: %s", devices[d], msg[d].c_str());
    return ok();
}

FG_EXPORT int fg_selftest_timeout(int limit_us)
{
    if (limit_us < 100 || limit_us > 1000000)
        return fail(FG_ERR_INVALID, "limit_us must be in [100, 1000000]");
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    std::lock_guard<std::mutex> lk(c->mu);
    if ((st = enter_stream(c, c->stream))) return st;
    // a small BF16 chain: B 64 x 512, A1 256 x 64, A2 128 x 256 (values irrelevant)
    const long N = 512, K1 = 64;
    const long M[2] = {256, 128}, K[2] = {K1, 256};
    const size_t need = carve_size((size_t)K1 * N * 2) + carve_size((size_t)M[0] * K[0] * 2) +
                        carve_size((size_t)M[1] * K[1] * 2) + carve_size((size_t)M[1] * N * 4) +
                        chain_scratch(FG_DT_BF16, 0, N, 2, M, K) + 4096;
    if ((st = arena_reserve(c, need))) return st;
    void *b = arena_take(c, (size_t)K1 * N * 2);
    void *a0 = arena_take(c, (size_t)M[0] * K[0] * 2);
    void *a1 = arena_take(c, (size_t)M[1] * K[1] * 2);
    void *cc = arena_take(c, (size_t)M[1] * N * 4);
    CUDA_TRY(cudaMemsetAsync(c->arena, 0, c->arena_off, c->stream));
    const Mat a[2] = {{a0, K[0]}, {a1, K[1]}};
    std::vector<StageArgs> stages;
    if ((st = build_tc_stages(c, FG_DT_BF16, FG_SEM_REF, cc, N, Mat{b, N}, N, 2, a, M, K,
                              nullptr, stages)))
        return st;
    int *done = nullptr;
    if ((st = take_counters(c, 3 * chain_counter_ints(2, M, N), &done))) return st;
    if ((st = launch(launch_tc_chain_stuck(stages.data(), done, c->status, c->sms,
                                           (unsigned long long)limit_us * 1000ull, c->stream),
                     "time-out self-test")))
        return st;
    // the kernel has returned on its own once this completes
    return collect_status(c);
}

FG_EXPORT int fg_profile_begin(void)
{
    DevCtx *c;
    int st;
    if ((st = get_ctx(&c))) return st;
    std::lock_guard<std::mutex> lk(c->mu);
    CUDA_TRY(cudaStreamSynchronize(c->work));
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
    CUDA_TRY(cudaStreamSynchronize(c->work));
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
    if ((st = enter_stream(c, user_stream(stream)))) return st;
    if ((st = arena_reserve(c, need))) return st;
    Mat b{B, N};
    if (pad_b) {
        void *p = arena_take(c, (size_t)K[0] * ldN * elt);
        CUDA_TRY(cudaMemcpy2DAsync(p, ldN * elt, B, N * elt, N * elt, K[0], cudaMemcpyDeviceToDevice,
                                   c->work));
        b = Mat{p, ldN};
    }
    if ((st = run_chain(c, dtype, semantics(), algo, C, N, b, N, num_gemm, a.data(), M.data(),
                        K.data(), pw.data())))
        return st;
    return ok();
}
