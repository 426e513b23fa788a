// The serving loop (flashgemm_b200.h, fg_server_*): chain requests on
// registered weights admitted in arrival order by a device-memory budget,
// packed into grouped launches (the executor of fg_group_api.cu) on a few
// streams so that batches overlap on the device, with latency statistics.
// Host code only.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "fg_host.h"

using namespace fg;
using namespace fg::host;

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
    long long next_id = 0, submitted = 0, completed = 0, failed = 0, shed = 0, batches = 0,
              batched = 0;
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
        if (s->o.max_queue_us > 0) {
            // load shedding: requests queued past their deadline are not run
            const double t = now_us();
            bool any = false;
            while (!s->pending.empty() && t - s->pending.front()->t_submit > s->o.max_queue_us) {
                fg_server_s::Req *q = s->pending.front();
                s->pending.pop_front();
                q->done = true;
                q->status = FG_ERR_BUSY;
                q->latency_us = t - q->t_submit;
                ++s->shed;
                any = true;
            }
            if (any) s->cv_done.notify_all();
        }
        if (s->pending.empty() || s->free_slots.empty()) {
            // a slot frees when a batch completes; with shedding on, wake in time
            // to shed the oldest request at its deadline
            long wait_us = 5000;
            if (s->o.max_queue_us > 0 && !s->pending.empty()) {
                const double left = s->o.max_queue_us - (now_us() - s->pending.front()->t_submit);
                wait_us = std::max(1l, std::min(wait_us, (long)left + 1));
            }
            s->cv_dispatch.wait_for(lk, std::chrono::microseconds(wait_us));
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
    while (s->completed + s->failed + s->shed < s->submitted) s->cv_done.wait(lk);
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
    out->shed = s->shed;
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
    s->submitted -= s->completed + s->failed + s->shed;
    s->completed = s->failed = s->shed = 0;
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
