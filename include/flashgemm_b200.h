/* flashgemm-b200 extension API.
 *
 * Everything here is new relative to the reference (whose API is the four
 * symbols of flashgemm.h and the LibShalom entry points of libshalom.h): error
 * reporting, the semantics and FP32-algorithm switches, and entry points that
 * take device pointers and a CUDA stream. No torch types: plain pointers,
 * sizes and a stream handle passed as void* (a cudaStream_t; NULL means CUDA's
 * legacy default stream).
 */
#ifndef FLASHGEMM_B200_EXT_H
#define FLASHGEMM_B200_EXT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    FG_OK = 0,
    FG_ERR_INVALID = 1,     /* bad shape, pointer or argument */
    FG_ERR_UNSUPPORTED = 2, /* valid for the reference but not handled here */
    FG_ERR_CUDA = 3,        /* a CUDA runtime call failed */
    FG_ERR_NO_DEVICE = 4,   /* no usable sm_100 device */
    FG_ERR_TIMEOUT = 5,     /* a kernel's bounded pipeline wait ran out */
    FG_ERR_NOMEM = 6,       /* device scratch allocation failed */
    FG_ERR_BUSY = 7         /* serving: the request was shed (queued past max_queue_us) */
} fg_status;

/* Status and message of the last call made on this host thread. */
int fg_last_status(void);
const char *fg_last_error(void);

/* Chain semantics.
 * FG_SEM_REF  (default): what the reference computes. BF16 and INT8 chains
 *   apply the reference's between-stage panel permutation (its stage output is
 *   stored row-major and re-read as K-pair / K-quad interleaved packed B,
 *   multigemm/src/kernel_bf16.h:6-32 + :356-391, kernel_int8.h:6-50 +
 *   :329-385), INT8 tail rows 12*floor(M/12) <= m < 4*floor(M/4) use the
 *   reference's shifted k-quad pairing, and INT8 rows m >= 4*floor(M/4) of C
 *   are left untouched.
 * FG_SEM_MATH: the mathematical chain with the same narrowing points (BF16 RNE,
 *   INT8 signed saturation) and no permutation.
 * The environment variable FG_SEMANTICS=ref|math sets the initial value. */
enum { FG_SEM_REF = 0, FG_SEM_MATH = 1 };
void fg_set_semantics(int sem);
int fg_get_semantics(void);

/* FP32 GEMM algorithm, separately for the chain and for LibShalom SGEMM.
 * FG_F32_FFMA:   plain FP32 FMA on the CUDA cores, bit-identical to the
 *                reference (default for LibShalom_sgemm_mp).
 * FG_F32_3XTF32: split-precision 3xTF32 on the tensor cores: each operand
 *                x = hi + lo (both TF32, round to nearest even), product
 *                hi*hi + hi*lo + lo*hi accumulated in FP32 (default for the chain).
 * Environment: FG_F32_ALGO / FG_SGEMM_ALGO = ffma|3xtf32. */
enum { FG_F32_FFMA = 0, FG_F32_3XTF32 = 1 };
void fg_set_f32_algo(int algo);
int fg_get_f32_algo(void);
void fg_set_sgemm_algo(int algo);
int fg_get_sgemm_algo(void);

/* How BF16 / INT8 chains are launched.
 * FG_CHAIN_FUSED (default): the whole chain in one persistent launch; a stage
 *   starts on a 256-column block as soon as the previous stage has stored it
 *   (or, where the library's schedule estimate prefers it, streams: it loads
 *   each 256-row tile of its input once that tile is stored; FG_CHAIN_STREAM=0
 *   or 1 forces either; the arithmetic and the results are the same).
 * FG_CHAIN_PER_GEMM: one tensor-core launch per GEMM, the plain per-GEMM path
 *   (same kernels' arithmetic, so the same results).
 * The environment variable FG_FUSED=0 selects the per-GEMM path initially. */
enum { FG_CHAIN_FUSED = 0, FG_CHAIN_PER_GEMM = 1 };
void fg_set_chain_mode(int mode);
int fg_get_chain_mode(void);

/* Fused BF16 / INT8 chains whose intermediates have at most 256 rows can keep
 * them on chip (the narrow chain kernel: one CTA per 128-column block, each
 * intermediate narrowed and permuted straight into shared memory; same
 * results as the other paths).
 * FG_NARROW_AUTO (default): where it is measured faster: every INT8 chain, and
 *   BF16 chains with at least one 128-column block per two SMs.
 * FG_NARROW_ALWAYS: every such chain.  FG_NARROW_OFF: never.
 * The environment variable FG_NARROW (0 / 1 / auto) sets the initial mode. */
enum { FG_NARROW_OFF = 0, FG_NARROW_ALWAYS = 1, FG_NARROW_AUTO = 2 };
void fg_set_narrow(int mode);
int fg_get_narrow(void);

/* Element types of a chain. */
enum { FG_DT_F32 = 0, FG_DT_BF16 = 1, FG_DT_INT8 = 2 };

/* Chain on device memory of the current device, same shapes and semantics as
 * the flashgemm_multi_* entry points: A[i] is M[i] x K[i] with leading
 * dimension K[i], B is K[0] x N and C is M[n-1] x N, both with leading
 * dimension N. C is float (FG_DT_F32, FG_DT_BF16) or int32 (FG_DT_INT8).
 * Asynchronous with respect to the host: ordered after the work already on
 * `stream`, and work later put on `stream` is ordered after it. Returns a
 * fg_status; errors that only a kernel can see (bounded waits that ran out)
 * show up in fg_sync(). */
int fg_chain_dev(int dtype, void *C, const void *B, long N, int num_gemm, const void *const *A,
                 const long *M, const long *K, void *stream);

/* C = A * B on device memory (row-major, dense leading dimensions), with the
 * given FP32 algorithm (FG_F32_FFMA or FG_F32_3XTF32). Asynchronous like
 * fg_chain_dev. */
int fg_sgemm_dev(float *C, const float *A, const float *B, long M, long N, long K, int algo,
                 void *stream);

/* Weight registry: weights copied once to the current device in the layout
 * the kernels read (16-byte rows), with their derived forms prepared once
 * (FP32: the 3xTF32 hi/lo split; INT8: the reference's shifted tail-row
 * block), so chains on them skip every per-call weight preparation. A is
 * M x K row-major (leading dimension K) in host (FG_MEM_HOST) or device
 * (FG_MEM_DEVICE) memory; a device source is read after the device is idle
 * (cudaDeviceSynchronize), so work on any stream that writes it is complete.
 * Blocking. */
typedef struct fg_weights_s *fg_weights;
enum { FG_MEM_HOST = 0, FG_MEM_DEVICE = 1 };
int fg_weights_register(int dtype, const void *A, long M, long K, int where, fg_weights *out);
/* Device bytes a registered weight set holds. */
long fg_weights_bytes(fg_weights w);
/* Waits for the device to be idle, then frees the weights. */
int fg_weights_release(fg_weights w);

/* Chain on registered weights (W[i] gives M_i, K_i; K_{i+1} must equal M_i):
 * device B (K_0 x N) and C (M_{n-1} x N), like fg_chain_dev. */
int fg_chain_registered(int dtype, void *C, const void *B, long N, int num_gemm,
                        const fg_weights *W, void *stream);

/* One chain of a grouped launch: device B (K_0 x N) and C (M_{n-1} x N) with
 * dense rows (N * element size a multiple of 16 bytes), registered weights. */
typedef struct {
    void *C;
    const void *B;
    long N;
    int num_gemm;
    const fg_weights *W;
} fg_chain_desc;

/* Many independent chains of one dtype in one grouped launch. BF16 / INT8 /
 * FP32-3xTF32: one persistent tensor-core kernel; every CTA (or CTA pair) of
 * the grid walks its share of all chains' tiles under a schedule the host
 * computes per shape set, and a tile of a chain's next stage starts as soon as
 * the column block it reads is complete. FP32 with FG_F32_FFMA: one grouped
 * CUDA-core launch per chain depth. Chains of uneven lengths and shapes mix
 * freely; results are bit-identical to running each chain alone with the same
 * kernel choice. The kernel and stage order come from fg_set_group_config (by
 * default the autotuner's choice). Asynchronous, ordered on `stream` like
 * fg_chain_dev. Corresponds to no reference entry point (the reference runs
 * one chain per call, multigemm/src/flashgemm.c:46). */
int fg_chain_group(int dtype, int nchains, const fg_chain_desc *chains, void *stream);

/* Kernel of a grouped launch. */
enum {
    FG_GROUP_AUTO = -1,      /* autotuned: measured choice for the shape set, else the cost model */
    FG_GROUP_PAIR = 0,       /* BF16 / INT8: CTA pairs (cta_group::2), 256 x 256 tiles, 6-stage ring */
    FG_GROUP_SINGLE_256 = 1, /* BF16 / INT8: single CTAs, 128 x 256 tiles, 4-stage ring */
    FG_GROUP_SINGLE_128 = 2  /* BF16 / INT8: single CTAs, 128 x 128 tiles, 6-stage ring;
                                FP32 3xTF32: 128 x 128 tiles, 3-stage ring (its only kernel) */
};
/* Stage order of a grouped launch. */
enum {
    FG_ORDER_AUTO = -1,
    FG_ORDER_FUSED = 0,  /* one launch; intermediates handed over per column block through L2 */
    FG_ORDER_LEVELS = 1  /* one launch per chain depth; each level spills its outputs to HBM */
};
/* Process-wide choice for later groups and plans (FG_GROUP_AUTO / FG_ORDER_AUTO:
 * the autotuner decides). */
void fg_set_group_config(int kernel, int order);
void fg_get_group_config(int *kernel, int *order);

/* A planned grouped launch, bound to its chains' buffers: tables, schedule and
 * intermediate buffers are built and uploaded once, so a launch is kernel
 * launches only and can be captured in a CUDA graph. */
typedef struct fg_plan_s *fg_plan;
int fg_plan_create(int dtype, int nchains, const fg_chain_desc *chains, fg_plan *out);
/* Stream-ordered launches of the plan on `stream` (NULL: legacy default stream). */
int fg_plan_launch(fg_plan plan, void *stream);
/* The first call captures fg_plan_launch into a CUDA graph; every call
 * launches that graph on `stream` (one launch for the whole group). */
int fg_plan_launch_graph(fg_plan plan, void *stream);
/* The plan's kernel and order (resolved), device bytes it owns, kernels per
 * launch, and total GEMM FLOPs. Any pointer may be NULL. */
int fg_plan_info(fg_plan plan, int *kernel, int *order, long *device_bytes, int *kernels,
                 double *flops);
/* Waits for the device to be idle, then frees the plan. */
int fg_plan_release(fg_plan plan);

/* Autotuner: times every (kernel, order) candidate on this group (`iters` timed
 * launches each after one warm-up, CUDA events on a private stream, buffers
 * overwritten) and remembers the fastest for the group's shape signature,
 * which FG_GROUP_AUTO groups of the same shapes then use. Outputs may be NULL. */
int fg_autotune_group(int dtype, int nchains, const fg_chain_desc *chains, int iters,
                      int *kernel, int *order, double *best_ms);
/* Remembered choices to / from a text file (one line per shape signature). */
int fg_autotune_save(const char *path);
int fg_autotune_load(const char *path);
/* Choice for a group without measuring (remembered, else the cost model). */
int fg_group_choice(int dtype, int nchains, const fg_chain_desc *chains, int *kernel, int *order);

/* ---------------------------------------------------------------- serving loop
 *
 * A request loop on the current device: chain requests on registered (resident)
 * weights are admitted in arrival order while the device-memory budget and a
 * launch slot allow, packed into grouped launches (one per dtype present) and
 * run on one of `slots` streams, so a batch admitted while others are still on
 * the GPU overlaps with them (each batch's persistent grid is capped at
 * SMs / slots CTAs unless ctas_per_batch says otherwise). The device is never
 * left idle while requests wait: a batch is launched at once when no other is
 * in flight, else when it holds max_batch requests or its oldest request has
 * waited max_wait_us. Results are the ones fg_chain_registered gives for the
 * same request with the same kernel choice. The reference has no serving
 * loop; this corresponds to none of its entry points. */
typedef struct fg_server_s *fg_server;
typedef struct {
    long long hbm_budget;  /* device bytes for requests' activations, intermediates and
                              tables (0: 80% of the free memory at creation) */
    int max_batch;         /* requests per batch (0: 64) */
    int slots;             /* batches in flight at once (0: 2) */
    int max_wait_us;       /* batching window while the device is busy (0: 200) */
    int ctas_per_batch;    /* grid cap of a batch's grouped kernels (0: SMs / slots) */
    int max_queue_us;      /* load shedding: a request still queued (not yet admitted)
                              this long after its submit is completed with FG_ERR_BUSY
                              instead of run, so that under overload the latency of the
                              requests that are served stays bounded (0: never shed) */
} fg_server_opts;

typedef struct {
    int dtype;              /* FG_DT_*; FP32 runs with the current fg_get_f32_algo() */
    int num_gemm;
    const fg_weights *W;    /* registered weights, K_{i+1} = M_i (copied at submit) */
    long N;                 /* activation columns; N * element size a multiple of 16 bytes */
    const void *B;          /* K_0 x N row-major activations */
    void *C;                /* M_{n-1} x N row-major result */
    int where;              /* FG_MEM_HOST: B and C are host memory (copied in and out
                               inside the request's latency; pinned memory copies
                               asynchronously); FG_MEM_DEVICE: device memory, used in place */
} fg_request;

typedef struct {
    long long submitted, completed, failed;
    long long shed;         /* requests completed with FG_ERR_BUSY (max_queue_us) */
    long long batches;      /* batches launched */
    double mean_batch;      /* requests per batch */
    double p50_us, p99_us, mean_us, max_us;  /* latency, submit to completion */
    double flops;           /* GEMM FLOPs of completed requests */
    double span_s;          /* first submit to last completion */
    long long peak_bytes;   /* most device bytes held by admitted requests at once */
} fg_server_stats;

int fg_server_create(const fg_server_opts *opts, fg_server *out);
/* Queues a request; returns its id (>= 0) or a negative fg_status. The request's
 * buffers must stay valid until fg_server_wait returns for it. Thread-safe. */
long long fg_server_submit(fg_server s, const fg_request *r);
/* Blocks until request `id` is done; its latency in microseconds (may be NULL).
 * Returns the request's status; the id is then forgotten. */
int fg_server_wait(fg_server s, long long id, double *latency_us);
/* Trace replay: submits reqs[i] at at_us[i] microseconds after the call (offsets
 * non-decreasing), from the calling thread, and stores the ids in ids[i] (a
 * negative fg_status where a submit was refused). Returns once all are
 * submitted, not done: a load generator for measuring the loop under a given
 * arrival process. */
int fg_server_replay(fg_server s, const fg_request *reqs, int n, const double *at_us,
                     long long *ids);
/* Blocks until every submitted request is done. */
int fg_server_drain(fg_server s);
int fg_server_get_stats(fg_server s, fg_server_stats *out);
/* Clears the latency record and counters (between the points of a rate sweep). */
int fg_server_reset_stats(fg_server s);
/* Drains, stops the loop's threads and frees its device memory. */
int fg_server_destroy(fg_server s);

/* Wait for all of the library's work on the current device and report any
 * kernel-side error since the last fg_sync (then cleared). This includes a
 * time-out of a fg_chain_bf16_noalloc call made with status == NULL, once the
 * caller's stream has finished that call. */
int fg_sync(void);

/* One chain split across GPUs, no collective. No counterpart in the reference,
 * which splits N across the OpenMP threads of one call (flashgemm.c:40-52,
 * :109-123); here the parts are devices. The arguments are those of the
 * reference entry points (host pointers; A, M, K as arrays of num_gemm) plus
 * the devices to use. Columns are cut on 32-column panel boundaries
 * (fg_split_columns), so every part runs the unchanged chain on its slice of B
 * and writes its slice of C, and the result is bit for bit the single-device
 * one. Blocking; one host thread per part. A device listed twice runs its
 * parts one after the other. */
int fg_chain_multi_device(int dtype, void *C, const void *B, long N, int num_gemm,
                          const void *const *A, const long *M, const long *K, int ndev,
                          const int *devices);

/* Columns [*c0, *c1) of N that part `index` of `parts` owns in
 * fg_chain_multi_device (and a rank of `parts` ranks in a column-partitioned
 * run): whole 32-column panels, as even as the panel count allows. Host
 * arithmetic only; needs no device. */
int fg_split_columns(long N, int parts, int index, long *c0, long *c1);

/* Self-test of failure detection; no counterpart in the reference (whose
 * only error path is print-and-return). Runs a small fused BF16 chain in which
 * the second stage waits on a dependency that nothing releases, with every
 * bounded wait of that one launch limited to limit_us microseconds (100 ..
 * 1000000). The waits run out, the kernel records the cause in the device
 * status word, stops its pipelines, frees its tensor memory and returns; this
 * call then returns what the host read: FG_ERR_TIMEOUT (message in
 * fg_last_error) when detection works. Nothing faults or hangs, and later calls
 * on the device run normally (the limit is restored in stream order). */
int fg_selftest_timeout(int limit_us);

/* Number of kernels this library has launched in this process (all devices).
 * Lets a benchmark count its own launches. */
unsigned long long fg_kernel_launches(void);

/* Per-launch device timing. While profiling is on, every kernel the library
 * launches on the current device is bracketed by CUDA events on the stream it
 * runs on. fg_profile_query sums, for one kernel class (or -1 for all), the
 * device time in ms, the number of launches and the algorithmic FLOPs
 * (2*M*N*K per GEMM stage). */
enum {
    FG_PK_TC_BF16 = 0,   /* tensor-core stage, BF16 */
    FG_PK_TC_I8 = 1,     /* tensor-core stage, INT8 */
    FG_PK_TC_TF32X3 = 2, /* tensor-core stage, 3xTF32 */
    FG_PK_FFMA = 3,      /* CUDA-core FP32 GEMM */
    FG_PK_AUX = 4        /* splits, weight preparation */
};
int fg_profile_begin(void);
int fg_profile_end(void);
int fg_profile_query(int kind, double *total_ms, unsigned long long *launches, double *flops);

/* Size of the fixed device array fg_chain_bf16_noalloc keeps its
 * between-stage buffers in: 48 MiB, present on every GPU that loads the library
 * until the process exits. */
#define FG_NOALLOC_SCRATCH_BYTES (48u << 20)

/* BF16 chain that allocates no device memory. No counterpart in the reference
 * (whose chain allocates and frees host scratch on every call).
 *
 * For callers that cannot call cudaMalloc when they run a chain: a framework
 * whose device memory all belongs to its own pool, a serving process that must
 * not grow its footprint after start-up. Same operands and semantics as
 * fg_chain_dev(FG_DT_BF16, ...) (device pointers: B K[0] x N, A[i] M[i] x K[i],
 * C M[n-1] x N float, dense rows), but the between-stage activations live in a
 * fixed array of FG_NOALLOC_SCRATCH_BYTES inside the library, and the kernels
 * run directly on `stream` (NULL: the legacy default stream). Nothing is
 * allocated or freed: no cudaMalloc, no cudaFree, no allocating library call.
 *
 * Limits: the largest two intermediates of alternating stages, each
 * M_i x round_up(N, 16) BF16 values, must fit in the array together
 * (FG_ERR_INVALID with the sizes otherwise; e.g. N = 4096 with widths
 * 4096 and 1024 needs 40 MiB); N and every K must be multiples of 8 and all
 * pointers 16-byte aligned.
 *
 * The array is shared by every call on a device and keeps the last call's
 * contents: calls whose kernels overlap on the GPU race, so order them (one
 * stream, or events). `status`, if not NULL, is a device int the kernels set
 * to a nonzero code when a bounded pipeline wait runs out (the caller clears
 * it). With NULL they set a word of the array instead, which is zero at load
 * and stays set until fg_sync() reports it as FG_ERR_TIMEOUT and clears it
 * (after the caller's stream has finished the call); the call itself returns
 * before its kernels run, so it cannot report a time-out in its return code.
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and the SM count; make that first call before any
 * stream capture. Returns a fg_status; the message is in fg_last_error(). */
int fg_chain_bf16_noalloc(float *C, const uint16_t *B, long N, int num_gemm,
                          const uint16_t *const *A, const long *M, const long *K, int *status,
                          void *stream);

/* Library version string. */
const char *fg_version(void);

#ifdef __cplusplus
}
#endif

#endif
