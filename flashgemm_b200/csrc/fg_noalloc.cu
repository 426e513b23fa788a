// BF16 chain without any device allocation: fg_chain_bf16_noalloc.
//
// Some callers cannot call cudaMalloc at the point where they run a chain: a
// host framework whose memory is owned by its own pool and that forbids any
// other allocation on the device, a serving process that must never grow its
// footprint after start-up, code that runs while another component holds the
// allocator. fg_chain_dev allocates its between-stage buffers from a scratch
// arena that it grows with cudaMalloc on demand; this entry point instead keeps
// them in one fixed array, fg_noalloc_scratch below, that is part of the
// library image. The caller passes inputs and outputs as before; nothing is
// allocated or freed during the call.
//
// The array occupies FG_NOALLOC_SCRATCH_BYTES of device memory on every GPU
// that loads the library, until the process exits. All calls on a device share
// it and it keeps the last call's contents, so two calls whose kernels overlap
// on the GPU (different streams, or different host threads without ordering)
// race on it; the caller orders them. Nothing in the array needs to start at
// zero: the between-stage buffers are written before they are read, and the
// array's status word (used when the caller passes status == NULL) is zero at
// load, only ever set by a kernel whose pipeline wait ran out, and read and
// cleared by fg_sync() (fg_noalloc_take_status below).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/flashgemm_b200.h"
#include "fg_kernels.h"

namespace fg {
int api_fail(int status, const char *msg);  // sets fg_last_status / fg_last_error (fg_api.cu)
int api_ok();
}  // namespace fg

namespace {

constexpr size_t kScratchBytes = FG_NOALLOC_SCRATCH_BYTES;
constexpr size_t kHeaderBytes = 256;  // [0, 4): kernel status word (used when status == NULL)

static __device__ __align__(256) unsigned char fg_noalloc_scratch[kScratchBytes];

struct DevScratch {
    char *base = nullptr;  // device address of fg_noalloc_scratch on this device
    int sms = 0;
};

std::mutex g_mu;
DevScratch g_dev[64];

// Once per device, with that device current: the device address of the array
// (its name in host code is only a host-side stand-in) and the SM count.
int setup(int dev, DevScratch *out)
{
    std::lock_guard<std::mutex> lk(g_mu);
    DevScratch &d = g_dev[dev];
    if (!d.base) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, fg_noalloc_scratch);
        if (e != cudaSuccess) {
            char msg[256];
            snprintf(msg, sizeof msg, "cudaGetSymbolAddress(fg_noalloc_scratch): %s",
                     cudaGetErrorString(e));
            return fg::api_fail(FG_ERR_CUDA, msg);
        }
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return fg::api_fail(FG_ERR_CUDA, cudaGetErrorString(e));
        d.sms = sms;
        d.base = static_cast<char *>(p);
    }
    *out = d;
    return FG_OK;
}

inline long round_up(long x, long a) { return (x + a - 1) / a * a; }

}  // namespace

namespace fg {
// Read and clear the array's status word on the current device, where this
// entry point has run on it (else 0). Synchronous copies on the legacy default
// stream: the caller has waited for the stream its chains ran on. Used by
// fg_sync(), so that a time-out of a call made with status == NULL is reported.
int noalloc_take_status(int dev, int *code)
{
    *code = 0;
    if (dev < 0 || dev >= 64) return 0;
    char *base;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        base = g_dev[dev].base;
    }
    if (!base) return 0;
    int v = 0;
    cudaError_t e = cudaMemcpy(&v, base, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && v != 0) e = cudaMemset(base, 0, sizeof(int));
    if (e != cudaSuccess) return (int)e;
    *code = v;
    return 0;
}
}  // namespace fg

extern "C" __attribute__((visibility("default"))) int fg_chain_bf16_noalloc(
    float *C, const uint16_t *B, long N, int num_gemm, const uint16_t *const *A, const long *M,
    const long *K, int *status, void *stream)
{
    char msg[256];
    if (!C || !B || !A || !M || !K) return fg::api_fail(FG_ERR_INVALID, "null pointer");
    if (num_gemm < 1 || num_gemm > 64)
        return fg::api_fail(FG_ERR_INVALID, "num_gemm must be in [1, 64]");
    if (N <= 0 || N % 8)
        return fg::api_fail(FG_ERR_INVALID, "N must be a positive multiple of 8 (16-byte rows)");
    if (N > (1l << 30)) return fg::api_fail(FG_ERR_INVALID, "N must be at most 2^30");
    if (((uintptr_t)C | (uintptr_t)B) & 15)
        return fg::api_fail(FG_ERR_INVALID, "B and C must be 16-byte aligned device pointers");
    for (int i = 0; i < num_gemm; ++i) {
        if (!A[i] || ((uintptr_t)A[i] & 15))
            return fg::api_fail(FG_ERR_INVALID, "weights must be 16-byte aligned device pointers");
        if (M[i] <= 0 || K[i] <= 0 || M[i] > (1l << 30) || K[i] > (1l << 30))
            return fg::api_fail(FG_ERR_INVALID, "M and K must be positive");
        if (K[i] % 8) {
            snprintf(msg, sizeof msg, "gemm %d: K must be a multiple of 8 (16-byte weight rows)",
                     i + 1);
            return fg::api_fail(FG_ERR_INVALID, msg);
        }
        if (i > 0 && K[i] != M[i - 1]) {
            snprintf(msg, sizeof msg, "gemm %d: K (%ld) must equal the previous M (%ld)", i + 1,
                     K[i], M[i - 1]);
            return fg::api_fail(FG_ERR_INVALID, msg);
        }
    }
    // Between-stage buffers alternate between two regions of the array: region
    // r holds the outputs of stages i with i % 2 == r (BF16, K_{i+1} x ldN).
    const long ldN = round_up(N, 16);
    size_t region[2] = {0, 0};
    for (int i = 0; i + 1 < num_gemm; ++i) {
        const size_t b = ((size_t)M[i] * ldN * 2 + 255) & ~(size_t)255;
        if (b > region[i & 1]) region[i & 1] = b;
    }
    const size_t need = kHeaderBytes + region[0] + region[1];
    if (need > kScratchBytes) {
        snprintf(msg, sizeof msg,
                 "chain needs %zu bytes of between-stage scratch; this entry point has %zu "
                 "(FG_NOALLOC_SCRATCH_BYTES); use fg_chain_dev",
                 need, kScratchBytes);
        return fg::api_fail(FG_ERR_INVALID, msg);
    }

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64)
        return fg::api_fail(FG_ERR_NO_DEVICE, "no CUDA device");
    DevScratch d;
    int st = setup(dev, &d);
    if (st) return st;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // status == NULL: the array's own word (zero at load; kernels only ever set
    // it, first time-out wins), kept until fg_sync() reads and clears it, so a
    // later call cannot erase an earlier call's time-out
    int *kstatus = status ? status : reinterpret_cast<int *>(d.base);
    uint16_t *buf[2] = {reinterpret_cast<uint16_t *>(d.base + kHeaderBytes),
                        reinterpret_cast<uint16_t *>(d.base + kHeaderBytes + region[0])};

    fg::StageArgs a;
    memset(&a, 0, sizeof a);
    a.op = fg::OP_BF16;
    a.N = (int)N;
    a.status = kstatus;
    a.permute = fg_get_semantics() == FG_SEM_REF ? 1 : 0;
    const void *x = B;
    long ldx = N;
    for (int i = 0; i < num_gemm; ++i) {
        const bool last = (i == num_gemm - 1);
        a.M = (int)M[i];
        a.K = (int)K[i];
        a.w = A[i];
        a.ld_w = K[i];
        a.x = x;
        a.ld_x = ldx;
        a.epi = last ? fg::EPI_F32 : fg::EPI_BF16;
        a.out = last ? static_cast<void *>(C) : static_cast<void *>(buf[i & 1]);
        a.ld_out = last ? N : ldN;
        a.m_written = (int)M[i];
        e = fg::launch_tc_stage(a, d.sms, s);
        if (e != cudaSuccess) return fg::api_fail(FG_ERR_CUDA, cudaGetErrorString(e));
        x = a.out;
        ldx = a.ld_out;
    }
    return fg::api_ok();
}
