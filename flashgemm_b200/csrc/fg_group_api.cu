// C ABI of grouped launches (flashgemm_b200.h): many chains of one dtype in
// one launch (fg_chain_group), plans built once and replayed through a CUDA
// graph (fg_plan_*), and the autotuner that chooses the grouped kernel and the
// stage order (fg_autotune_*, fg_set_group_config). Host code only; the
// serving loop (fg_serve.cu) builds its batches with the same executor.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "fg_host.h"

// ---------------------------------------------------------------- grouped launches

namespace fg {
namespace host {

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

bool panel_enabled()
{
    static const bool on = [] {
        const char *v = getenv("FG_PANEL");
        return !(v && v[0] == '0');
    }();
    return on;
}

int panel_finish(DevCtx *c, GroupExec &gx, int max_units)
{
    if (gx.panel.empty()) return FG_OK;
    int ctas = 0;
    cudaError_t e = panel_capacity(max_units > 0 ? max_units : c->sms, ctas);
    if (e != cudaSuccess) return fail(FG_ERR_CUDA, "panel launch: %s", cudaGetErrorString(e));
    std::vector<int> cost, nblocks;
    long total = 0;
    for (const PanelChain &pc : gx.panel) {
        int kb = 0;
        for (int i = 0; i < pc.n; ++i) kb += (pc.K[i] + 31) / 32;
        cost.push_back(kb);
        nblocks.push_back(panel_blocks_of(pc.N));
        total += nblocks.back();
    }
    if (total < ctas) ctas = (int)total;
    panel_plan(cost, nblocks, ctas, gx.panel_blocks, gx.panel_off);
    gx.panel_ctas = ctas;
    return FG_OK;
}

// Host side of a grouped launch: between-stage buffers carved from `cv`, stage
// lists, schedules and tables (device addresses of the tables come later).
int group_build(DevCtx *c, int dtype, int algo, int kernel, int order, int nchains,
                const fg_chain_desc *chains, Carver &cv, GroupExec &gx, int *status,
                int max_units)
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
        if (dtype == FG_DT_F32 && panel_enabled() && panel_eligible(N, n, M.data(), K.data()) &&
            gx.panel.size() < 65536) {
            // intermediates on chip: one panel launch for all such chains
            PanelChainArgs pa;
            memset(&pa, 0, sizeof pa);
            pa.n = n;
            pa.N = N;
            pa.B = (const float *)d.B;
            pa.ldb = N;
            pa.C = (float *)d.C;
            pa.ldc = N;
            for (int i = 0; i < n; ++i) {
                pa.w_hi[i] = pw[i].hi;
                pa.w_lo[i] = pw[i].lo;
                pa.ldw[i] = pw[i].ld_split;
                pa.M[i] = M[i];
                pa.K[i] = K[i];
                pa.kchunk[i] = tf32_chunk_blocks(K[i]);
            }
            PanelChain pc;
            cudaError_t e = panel_chain_desc(pa, pc);
            if (e != cudaSuccess)
                return fail(FG_ERR_INVALID, "chain %d: panel tables: %s", j, cudaGetErrorString(e));
            gx.panel.push_back(pc);
            for (int i = 0; i < n; ++i) gx.panel_flops += gemm_flops(M[i], N, K[i]);
            continue;
        }
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
    if (int st = panel_finish(c, gx, max_units)) return st;
    const int nlaunch = all.empty() ? 0 : order == FG_ORDER_LEVELS ? maxd + 1 : 1;
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
    b += carve_size(gx.panel.size() * sizeof(PanelChain)) +
         carve_size(gx.panel_blocks.size() * sizeof(uint32_t)) +
         carve_size(gx.panel_off.size() * sizeof(int));
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
    if (!gx.panel.empty()) {
        gx.panel_dev = (PanelChain *)cv.take(gx.panel.size() * sizeof(PanelChain));
        gx.panel_blocks_dev = (uint32_t *)cv.take(gx.panel_blocks.size() * sizeof(uint32_t));
        gx.panel_off_dev = (int *)cv.take(gx.panel_off.size() * sizeof(int));
    }
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
    if (!gx.panel.empty()) {
        CUDA_TRY(copy(gx.panel_dev, gx.panel.data(), gx.panel.size() * sizeof(PanelChain)));
        CUDA_TRY(copy(gx.panel_blocks_dev, gx.panel_blocks.data(),
                      gx.panel_blocks.size() * sizeof(uint32_t)));
        CUDA_TRY(copy(gx.panel_off_dev, gx.panel_off.data(), gx.panel_off.size() * sizeof(int)));
    }
    return FG_OK;
}

int group_launch(DevCtx *c, const GroupExec &gx, cudaStream_t s, bool capturing,
                 int *status)
{
    if (!status) status = c->status;
    if (!gx.panel.empty()) {
        int st = run_kernel_on(c, s, capturing, FG_PK_TC_TF32X3, gx.panel_flops,
                               "panel-resident chains", [&] {
            return launch_panel(gx.panel_dev, gx.panel_blocks_dev, gx.panel_off_dev, gx.panel_ctas,
                                status, s);
        });
        if (st) return st;
    }
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

}  // namespace host
}  // namespace fg

using namespace fg;
using namespace fg::host;

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
    // everything runs on the caller's stream, after all earlier library work
    if ((st = enter_stream(c, user_stream(stream)))) return st;
    if ((st = arena_reserve(c, group_buf_bytes(dtype, algo, nchains, chains)))) return st;
    Carver cb;
    cb.base = c->arena;
    GroupExec gx;
    if ((st = group_build(c, dtype, algo, kernel, order, nchains, chains, cb, gx))) return st;
    if ((st = tab_reserve(c, group_tab_bytes(gx)))) return st;
    Carver ct;
    ct.base = c->tab;
    group_place(gx, ct);
    if ((st = group_upload(gx, c->work, false))) return st;
    if ((st = group_launch(c, gx, c->work, false))) return st;
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
