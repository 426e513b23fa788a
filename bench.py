"""Benchmark of the flashgemm hot path on B200: one JSON line on stdout.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload all|bf16-chain|int8-chain|f32-gemm|bf16-gemm|int8-gemm|
                                f32-groups|serve]

By default (--workload all) the line's headline is the BF16 chain below, and
the same line carries the rest of the metric as sub-objects, each with its
own roofline, clocks, end-to-end figure and reference CPU baseline:
"int8_chain" (the INT8 chain of 4 GEMMs), "f32_gemm" (the 1024^3 FP32 SGEMM on
the plain FMA kernel), "f32_groups" (128 of the grouped FP32 chains, 2 of them
tall-skinny, as one graph-captured 3xTF32 launch) and "serve" (the serving
loop at 0.6 x its measured capacity, 4000 Poisson requests, p50/p99 latency),
plus "peaks_this_run" (cuBLAS BF16 / INT8 / TF32 / FP32 bursts at 8192^3, the
denominators the peaks file does not hold).

A step is one pass of the hot path over one batch: the BF16 chain
of three GEMMs C = A3*(A2*(A1*B)) with B 1024 x 4096 (the activations X
[4096 x 1024] of X*W1*W2*W3, in the reference's orientation) and weights
4096 x 1024, 1024 x 4096, 1024 x 1024, BF16 inputs, FP32 accumulation, BF16
intermediates with the reference's panel permutation, FP32 output. Inputs are
seeded synthetic data in HBM; L2 is flushed (a 256 MiB write) between timed
steps, outside each step's events.

Multi-GPU (torchrun, one process per GPU): the activation columns are
partitioned, so every rank runs its own full step on its own shard with no
data-path collective (weak scaling); NCCL carries only the barrier and the
max-over-ranks time.

--impl reference times the reference's own CPU implementation (compiled from
its sources into oracle/_ref) on this machine's host cores, on a bounded
column sample of the same workload, and prints the same line with
"impl": "reference".

--workload f32-groups: 512 independent FP32 chains (length 2-5, dimensions
log-uniform on multiples of 16 in [64, 4096], activation columns up to 8192,
plus tall-skinny chains of 65536 columns with 64 x 64 weights), N(0,1)/sqrt(K)
entries, run as one graph-captured grouped 3xTF32 launch; the same group
through the plain FP32 kernel beside it, and both errors against FP64 on a
seeded sample of the chains.

--workload serve: the library's serving loop under Poisson arrivals of chain
requests (length U{2..6}, dimensions and activation columns log-uniform on
multiples of 16 in [64, 4096], 50/30/20 BF16/INT8/FP32 over 64 resident
weight sets), replayed from native code at fractions of the capacity measured
on a burst; p50/p99 latency and throughput per rate.
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (dtype, N, K1, Ms)
    "bf16-chain": ("bf16", 4096, 1024, [4096, 1024, 1024]),
    "int8-chain": ("int8", 8192, 2048, [4096, 2048, 4096, 1024]),
    "f32-gemm": ("f32", 1024, 1024, [1024]),
    "bf16-gemm": ("bf16", 8192, 8192, [8192]),
    "int8-gemm": ("int8", 8192, 8192, [8192]),
}
DESCR = {
    "bf16-chain": "BF16 chain of 3 GEMMs: X[4096x1024]*W1[1024x4096]*W2[4096x1024]*W3[1024x1024]",
    "int8-chain": "INT8 chain of 4 GEMMs: X[8192x2048]*W1..W4, widths 2048->4096->2048->4096->1024",
    "f32-gemm": "single FP32 GEMM C=A*B, M=N=K=1024 (plain FP32 FMA kernel)",
    "bf16-gemm": "single BF16 GEMM (one-stage chain) M=N=K=8192, the shape of the cuBLAS peak",
    "int8-gemm": "single INT8 GEMM (one-stage chain) M=N=K=8192",
}


def flops_of(N, K1, Ms):
    Ks = [K1] + Ms[:-1]
    return sum(2.0 * N * m * k for m, k in zip(Ms, Ks))


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p, "measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, \
            "fallback"


# ---------------------------------------------------------------- clocks (NVML, read only)

class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


class ClockSampler:
    """Samples SM clock and clock-event reasons of one GPU every 10 ms."""

    REASONS = {
        "gpu_idle": 0x1, "applications_clocks_setting": 0x2, "sw_power_cap": 0x4,
        "hw_slowdown": 0x8, "sync_boost": 0x10, "sw_thermal_slowdown": 0x20,
        "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80,
    }

    def __init__(self, index):
        self.samples = []
        self.reasons = 0
        self.max_mhz = None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:  # noqa: BLE001 - clocks are reported as unavailable
            self._h = None

    def _run(self):
        while not self._stop.is_set():
            try:
                mhz = self._nv.nvmlDeviceGetClockInfo(self._h, self._nv.NVML_CLOCK_SM)
                r = self._nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                util = self._nv.nvmlDeviceGetUtilizationRates(self._h).gpu
                self.samples.append((mhz, r, util))
            except Exception:  # noqa: BLE001
                pass
            time.sleep(0.01)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        if self._h is not None:
            self._stop.set()
            self._t.join()

    def summary(self):
        if self._h is None or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"]}
        loaded = [s for s in self.samples if s[2] > 0] or self.samples
        mhz = statistics.median(s[0] for s in loaded)
        bits = 0
        for s in loaded:
            bits |= s[1]
        names = [k for k, v in self.REASONS.items() if bits & v and k != "gpu_idle"]
        return {"sm_mhz": mhz, "sm_max_mhz": self.max_mhz, "reasons": names,
                "samples": len(self.samples)}


# ---------------------------------------------------------------- CPU reference / port

def cpu_info():
    flags = set()
    model = ""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags") and not flags:
                    flags = set(line.split(":", 1)[1].split())
                if line.startswith("model name") and not model:
                    model = line.split(":", 1)[1].strip()
    except OSError:
        pass
    return flags, model


def reference_runner():
    """The reference's own implementation if it was built here and this CPU
    runs its instructions (AVX-512 F/BW, VNNI, BF16); else the C port."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    flags, model = cpu_info()
    need = {"avx512f", "avx512bw", "avx512_vnni", "avx512_bf16"}
    if oracle.ref_available() and need <= flags:
        return oracle, "reference", model, "amx_tile" in flags
    return oracle, "port", model, "amx_tile" in flags


def time_cpu(workload, steps=None, warmup=1, budget_s=12.0):
    """TFLOP/s of the reference (or port) on a column sample of the workload.

    steps=None: repeat for about budget_s seconds (the cpu_baseline leg).
    steps=K: exactly K timed steps, the column sample sized from one calibration
    call so that the K steps take about a minute in total.
    Returns (tflops, descr dict, per-step seconds)."""
    oracle, kind, model, amx = reference_runner()
    dt, N, K1, Ms = WORKLOADS[workload]
    threads = os.cpu_count() or 1

    def prepare(ns):
        if dt == "f32":
            A, Bm = oracle.sgemm_inputs(Ms[0], ns, K1, seed=1)

            def one():
                if kind == "reference":
                    oracle.ref_sgemm(A, Bm, threads=threads)
                else:
                    oracle.sgemm_f32(A, Bm)
        else:
            B, As, Ks = oracle.chain_inputs(dt, ns, K1, Ms, seed=1)

            def one():
                if kind == "reference":
                    oracle.ref_chain(dt, B, As, ns, Ms, Ks, threads=threads)
                else:
                    oracle.chain(dt, B, As, ns, Ms, Ks, mode=oracle.REF, threads=threads)
        return one

    ns = min(N, 512)
    one = prepare(ns)
    t0 = time.perf_counter()
    one()
    t_cal = time.perf_counter() - t0
    if steps is not None:
        per_step = 60.0 / max(steps + warmup, 1)
        ns = int(ns * per_step / max(t_cal, 1e-6)) // 32 * 32
        ns = max(32, min(N, ns))
        one = prepare(ns)
    for _ in range(warmup):
        one()
    times = []
    t_end = time.perf_counter() + budget_s
    while True:
        t0 = time.perf_counter()
        one()
        times.append(time.perf_counter() - t0)
        if steps is not None:
            if len(times) >= steps:
                break
        elif len(times) >= 3 and time.perf_counter() > t_end:
            break
    fl = flops_of(ns, K1, Ms)
    med = statistics.median(times)
    descr = {"kind": kind, "cores": threads, "cpu": model, "amx_available": amx,
             "amx_used": False,
             "sample": f"{ns} of {N} activation columns per step (work scales with columns), "
                       f"median of {len(times)} steps"}
    return fl / med / 1e12, descr, times


# ---------------------------------------------------------------- GPU arm

def make_inputs(dt, N, K1, Ms, seed):
    """Seeded synthetic operands (host numpy), same distributions as the tests:
    f32 U[-1, 1]; bf16 N(0,1)/sqrt(K) rounded to BF16; int8 U{-127..127}."""
    rng = np.random.default_rng(seed)
    Ks = [K1] + Ms[:-1]
    if dt == "f32":
        B = rng.uniform(-1, 1, (K1, N)).astype(np.float32)
        As = [rng.uniform(-1, 1, (m, k)).astype(np.float32) for m, k in zip(Ms, Ks)]
    elif dt == "bf16":
        def bf(x):
            u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
            return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
        B = bf(rng.standard_normal((K1, N)))
        As = [bf(rng.standard_normal((m, k)) / np.sqrt(k)) for m, k in zip(Ms, Ks)]
    else:
        B = rng.integers(-127, 128, size=(K1, N)).astype(np.int8).view(np.uint8)
        As = [rng.integers(-127, 128, size=(m, k)).astype(np.int8) for m, k in zip(Ms, Ks)]
    return B, As, Ks


# ---------------------------------------------------------------- grouped FP32 chains

GROUP_CHAINS = 512
GROUP_SKINNY = 8


def group_specs(seed, count=GROUP_CHAINS, skinny=GROUP_SKINNY):
    """(N, K1, [M_1..M_n]) of the grouped workload: chain length U{2..5},
    dimensions log-uniform on multiples of 16 in [64, 4096], activation columns
    log-uniform in [64, 8192], plus `skinny` chains of 65536 columns with 64 x 64
    weights; shuffled."""
    rng = np.random.default_rng(seed)

    def dim(lo, hi):
        v = int(16 * round(float(np.exp(rng.uniform(np.log(lo), np.log(hi)))) / 16))
        return min(max(v, lo), hi)

    specs = []
    for _ in range(count - skinny):
        n = int(rng.integers(2, 6))
        N = dim(64, 8192)
        dims = [dim(64, 4096) for _ in range(n + 1)]
        specs.append((N, dims[0], dims[1:]))
    for _ in range(skinny):
        n = int(rng.integers(2, 6))
        specs.append((65536, 64, [64] * n))
    order = rng.permutation(len(specs))
    return [specs[i] for i in order]


def group_sample(specs, seed, count=16, skinny=2, max_gflop=20.0):
    """Indices of the chains checked against FP64 and timed on the CPU."""
    rng = np.random.default_rng(seed)
    small = [i for i, (N, K1, Ms) in enumerate(specs)
             if N != 65536 and flops_of(N, K1, Ms) <= max_gflop * 1e9]
    thin = [i for i, (N, _, _) in enumerate(specs) if N == 65536]
    pick = list(rng.choice(small, size=min(count, len(small)), replace=False)) if small else []
    return sorted(int(i) for i in pick + thin[:skinny])


def group_cpu(specs, sample, host, steps=None, budget_s=12.0):
    """The reference's FP32 chain (or the C port) on the sampled chains, all
    host threads: TFLOP/s over the sample. steps=None: repeat for budget_s."""
    oracle, kind, model, amx = reference_runner()
    threads = os.cpu_count() or 1
    fl = sum(flops_of(*specs[i]) for i in sample)

    def one():
        for i in sample:
            N, K1, Ms = specs[i]
            B, As = host[i]
            Ks = [K1] + Ms[:-1]
            if kind == "reference":
                oracle.ref_chain("f32", B, As, N, Ms, Ks, threads=threads)
            else:
                oracle.chain("f32", B, As, N, Ms, Ks)
    one()
    times = []
    t_end = time.perf_counter() + budget_s
    while True:
        t0 = time.perf_counter()
        one()
        times.append(time.perf_counter() - t0)
        if steps is not None:
            if len(times) >= steps:
                break
        elif len(times) >= 3 and time.perf_counter() > t_end:
            break
    med = statistics.median(times)
    descr = {"kind": kind, "cores": threads, "cpu": model, "amx_available": amx,
             "amx_used": False,
             "sample": f"{len(sample)} of the group's {len(specs)} chains "
                       f"({fl / 1e9:.1f} GFLOP per step, all of each chain), median of "
                       f"{len(times)} steps"}
    return fl / med / 1e12, descr, times


def group_host_inputs(specs, indices, seed):
    """Host operands (B, [A_i]) of chosen chains with the workload's
    distributions, drawn on the host (chain j from seed + j): inputs for timing
    the CPU reference where no GPU drew them."""
    import torch
    out = {}
    for j in indices:
        N, K1, Ms = specs[j]
        g = torch.Generator().manual_seed(seed + j)
        Ks = [K1] + Ms[:-1]
        As = [(torch.randn(m, k, generator=g) / float(np.sqrt(k))).numpy() for m, k in zip(Ms, Ks)]
        B = torch.randn(K1, N, generator=g).numpy()
        out[j] = (np.ascontiguousarray(B), [np.ascontiguousarray(a) for a in As])
    return out


def run_groups(args, world, rank, local_rank, ctx=None):
    """Grouped FP32 chains. g: the shared GPU context (None: the reference arm).
    Returns the line (a dict) on rank 0 of our arm, else None."""
    seed = 4321
    n = max(8, args.group_chains)
    nsk = n if args.skinny_only else max(1, GROUP_SKINNY * n // GROUP_CHAINS)
    specs = group_specs(seed, count=n, skinny=nsk)
    sample = group_sample(specs, seed + 1)
    total_flops = sum(flops_of(*s) for s in specs)
    config = {"workload": f"{n} independent FP32 chains in one graph-captured grouped launch: "
                          "length U{2..5}, dims log-uniform on multiples of 16 in [64, 4096], "
                          f"activation columns log-uniform in [64, 8192], {nsk} tall-skinny chains "
                          "(65536 columns, 64 x 64 weights); N(0,1)/sqrt(K) entries",
              "chains": len(specs), "stages": sum(len(s[2]) for s in specs),
              "gflop_per_step_per_gpu": total_flops / 1e9,
              "l2": "flushed between steps (256 MiB write outside the step events)",
              "parallelism": f"dp{world} (each rank runs its own group, no collective)"}
    metric = "grouped FP32 chains TFLOP/s (3xTF32)"
    if args.impl == "reference":
        if rank != 0:
            return 0
        host = group_host_inputs(specs, sample, seed)
        tf, descr, times = group_cpu(specs, sample, host, steps=args.steps)
        return {"impl": "reference", "metric": metric, "value": tf, "unit": "TFLOP/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * statistics.median(times), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded)", "config": config,
                "cpu_baseline": dict(descr, value=tf, unit="TFLOP/s"),
                "e2e": {"value": tf, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}

    torch, fg, dist, dev = ctx.torch, ctx.fg, ctx.dist, ctx.dev
    # operands: weights registered once (resident), activations and outputs in HBM;
    # chain j draws from seed + j (+ rank offset), on the device
    chains = []
    host = {}  # the sampled chains' operands, copied back for the FP64 check
    t_gen = time.perf_counter()
    for j, (N, K1, Ms) in enumerate(specs):
        g = torch.Generator(device=dev).manual_seed(seed + j + 100000 * rank)
        Ks = [K1] + Ms[:-1]
        W, keep = [], []
        for m, k in zip(Ms, Ks):
            a = torch.randn(m, k, generator=g, device=dev) / float(np.sqrt(k))
            W.append(fg.Weights("f32", a))
            if j in sample:
                keep.append(a.cpu().numpy())
            del a
        B = torch.randn(K1, N, generator=g, device=dev)
        if j in sample:
            host[j] = (B.cpu().numpy(), keep)
        C = torch.empty(Ms[-1], N, device=dev)
        chains.append((C, B, N, W))
    t_gen = time.perf_counter() - t_gen
    weight_bytes = sum(w.nbytes for c in chains for w in c[3])
    flush = ctx.flush

    def timed(plan, sampler=None):
        for _ in range(max(args.warmup, 3)):
            plan.launch(graph=True)
        torch.cuda.synchronize(dev)
        fg.sync()
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
        l0 = fg.kernel_launches()
        with (sampler if sampler is not None else _Null()):
            for i in range(args.steps):
                flush.fill_(i & 0xFF)
                starts[i].record()
                plan.launch(graph=True)
                stops[i].record()
            torch.cuda.synchronize(dev)
        fg.sync()
        launches = fg.kernel_launches() - l0
        ms = sum(a.elapsed_time(b) for a, b in zip(starts, stops))
        if dist:
            t = torch.tensor([ms], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, launches

    def kernel_profile(plan, kind, n=5):
        """Average device time of the plan's main kernel, CUDA events on the
        stream it runs on (direct launches; a graph replay runs the same kernels)."""
        fg.profile_begin()
        for _ in range(n):
            flush.fill_(1)
            plan.launch(graph=False)
        torch.cuda.synchronize(dev)
        fg.sync()
        fg.profile_end()
        return fg.profile_query(kind)

    def sample_out():
        return {j: chains[j][0].cpu().numpy().copy() for j in sample}

    # ---- 3xTF32: autotuned stage order, one graph-captured launch per step
    fg.set_f32_algo("3xtf32")
    tune = fg.autotune_group("f32", chains, iters=2)
    plan = fg.Plan("f32", chains)
    info = plan.info()
    sampler = ClockSampler(torch.cuda.current_device())
    x3_ms, launches = timed(plan, sampler)
    k_ms, k_n, k_fl = kernel_profile(plan, fg.FG_PK_TC_TF32X3)
    out_x3 = sample_out()

    # ---- end to end: host activations in, host results out, every step
    e2e_steps = args.e2e_steps or 3
    hB = [torch.empty(tuple(c[1].shape), dtype=torch.float32, pin_memory=True) for c in chains]
    hC = [torch.empty(tuple(c[0].shape), dtype=torch.float32, pin_memory=True) for c in chains]
    for h, c in zip(hB, chains):
        h.copy_(c[1])

    def e2e_step():
        for h, c in zip(hB, chains):
            c[1].copy_(h, non_blocking=True)
        plan.launch(graph=True)
        for h, c in zip(hC, chains):
            h.copy_(c[0], non_blocking=True)
        torch.cuda.synchronize(dev)

    e2e_step()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    h2d = sum(h.numel() * 4 for h in hB)
    d2h = sum(h.numel() * 4 for h in hC)
    del hB, hC
    plan.release()

    # ---- plain FP32 (FFMA, one grouped launch per chain depth)
    fg.set_f32_algo("ffma")
    plan2 = fg.Plan("f32", chains)
    ff_ms, _ = timed(plan2)
    out_ff = sample_out()
    plan2.release()

    # ---- the tall-skinny chains alone: HBM-bound, so GB/s of their fused ideal
    # (B read once, C written once) against the measured HBM bandwidth
    thin = [j for j, sp in enumerate(specs) if sp[0] == 65536]
    skinny = None
    if thin:
        sub = [chains[j] for j in thin]
        sk_bytes = sum(4 * (specs[j][1] + specs[j][2][-1]) * specs[j][0] for j in thin)
        sk_fl = sum(flops_of(*specs[j]) for j in thin)
        skinny = {"chains": len(thin), "algorithmic_bytes_per_step": sk_bytes,
                  "gflop_per_step": sk_fl / 1e9}
        for algo in ("3xtf32", "ffma"):
            fg.set_f32_algo(algo)
            p = fg.Plan("f32", sub)
            for _ in range(3):
                p.launch(graph=True)
            torch.cuda.synchronize(dev)
            reps, tot = 10, 0.0
            for i in range(reps):
                flush.fill_(i & 0xFF)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                p.launch(graph=True)
                b.record()
                torch.cuda.synchronize(dev)
                tot += a.elapsed_time(b)
            fg.sync()
            p.release()
            ms = tot / reps
            key = "3xtf32" if algo == "3xtf32" else "plain"
            skinny[f"ms_{key}"] = ms
            skinny[f"gbs_{key}"] = sk_bytes / (ms / 1e3) / 1e9
    fg.set_f32_algo("3xtf32")
    for c in chains:
        for w in c[3]:
            w.release()
    if dist:
        dist.barrier()
    if rank != 0:
        return None

    # ---- accuracy against FP64 on the sample (host)
    err_x3, err_ff = [], []
    for j in sample:
        B, As = host[j]
        exact = B.astype(np.float64)
        for a in As:
            exact = a.astype(np.float64) @ exact
        nrm = np.linalg.norm(exact)
        err_x3.append(float(np.linalg.norm(out_x3[j] - exact) / nrm))
        err_ff.append(float(np.linalg.norm(out_ff[j] - exact) / nrm))
    ratio = [a / b for a, b in zip(err_x3, err_ff) if b > 0]

    value = world * total_flops * args.steps / (x3_ms / 1e3) / 1e12
    plain = world * total_flops * args.steps / (ff_ms / 1e3) / 1e12
    peaks, peak_src = load_peaks()
    if skinny:
        for key in ("3xtf32", "plain"):
            skinny[f"frac_hbm_{key}"] = skinny[f"gbs_{key}"] / peaks["hbm_gbs"]
        skinny["hbm_peak_gbs"] = peaks["hbm_gbs"]
        skinny["peak_source"] = f"hbm_gbs (STREAM-style copy); {peak_src}"
    peak = peaks.get("bf16_tflops") / 2.0 / 3.0
    achieved = k_fl / (k_ms / 1e3) / 1e12 if k_ms > 0 else None
    roofline = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak if achieved else None, "traffic": None,
                "kernel": "fg::tc_group_kernel<OP_TF32X3,128,3> (all chains, one launch per order level)",
                "launches_timed": k_n, "avg_launch_us": 1e3 * k_ms / k_n if k_n else None,
                "peak_source": "bf16_tflops / 2 (dense TF32 is half the BF16 rate) / 3 "
                               f"(three MMAs per 3xTF32 product); {peak_src}"}
    names = {0: "fused", 1: "levels"}
    line = {"metric": metric, "value": value, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": x3_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (3xTF32 split on tensor cores, FP32 accumulate)",
            "data": "synthetic (seeded; no dataset involved)", "config": config,
            "clocks": sampler.summary(), "gpu_launches": launches,
            "e2e": {"value": world * total_flops * e2e_steps / e2e_s / 1e12, "unit": "TFLOP/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                    "api": "fg_plan_launch_graph on registered weights; every chain's B copied "
                           "from pinned host memory and C copied back each step"},
            "roofline": roofline,
            "plain_fp32": {"value": plain, "unit": "TFLOP/s", "ms_per_step": ff_ms / args.steps,
                           "path": "grouped FFMA kernel, one launch per chain depth"},
            "x3_vs_plain": value / plain,
            "skinny": skinny,
            "accuracy": {"sample_chains": len(sample),
                         "rel_frob_vs_fp64_3xtf32_max": max(err_x3),
                         "rel_frob_vs_fp64_plain_max": max(err_ff),
                         "ratio_3xtf32_over_plain_max": max(ratio) if ratio else None},
            "plan": {"order": names.get(info["order"], info["order"]),
                     "autotune": {"order": names.get(tune[1], tune[1]), "ms": tune[2]},
                     "device_bytes": info["device_bytes"], "kernels_per_step": info["kernels"],
                     "weight_bytes": weight_bytes, "setup_s": t_gen}}
    if world == 1:
        tf, descr, _ = group_cpu(specs, sample, host, budget_s=args.cpu_budget)
        line["cpu_baseline"] = dict(descr, value=tf, unit="TFLOP/s")
    return line


# ---------------------------------------------------------------- serving stream

SERVE_SETS = 64
SERVE_MIX = (("bf16", 0.5), ("int8", 0.3), ("f32", 0.2))


def serve_sets(seed):
    """64 weight sets: dtypes in the 50/30/20 BF16/INT8/FP32 mix, chain length
    U{2..6}, dimensions log-uniform on multiples of 16 in [64, 4096]."""
    rng = np.random.default_rng(seed)
    counts = {"bf16": 32, "int8": 19, "f32": 13}
    dts = [d for d, c in counts.items() for _ in range(c)]
    rng.shuffle(dts)

    def dim():
        v = int(16 * round(float(np.exp(rng.uniform(np.log(64), np.log(4096)))) / 16))
        return min(max(v, 64), 4096)

    out = []
    for dt in dts:
        n = int(rng.integers(2, 7))
        dims = [dim() for _ in range(n + 1)]
        out.append((dt, dims[0], dims[1:]))
    return out


def serve_requests(seed, sets, count):
    """(set index, N) per request: dtype by the mix, a set of that dtype
    uniformly, N log-uniform on multiples of 16 in [64, 4096]."""
    rng = np.random.default_rng(seed)
    by = {d: [i for i, s in enumerate(sets) if s[0] == d] for d, _ in SERVE_MIX}
    dts = rng.choice([d for d, _ in SERVE_MIX], size=count, p=[p for _, p in SERVE_MIX])
    out = []
    for d in dts:
        i = int(rng.choice(by[str(d)]))
        N = int(16 * round(float(np.exp(rng.uniform(np.log(64), np.log(4096)))) / 16))
        out.append((i, min(max(N, 64), 4096)))
    return out


def serve_flops(sets, reqs):
    return [flops_of(N, sets[i][1], sets[i][2]) for i, N in reqs]


def serve_cpu(sets, reqs, host, steps=None, budget_s=12.0):
    """The reference's chains (or the C port) on sampled requests, all host threads."""
    oracle, kind, model, amx = reference_runner()
    threads = os.cpu_count() or 1
    fl = sum(serve_flops(sets, reqs))

    def one():
        for i, N in reqs:
            dt, K1, Ms = sets[i]
            B, As = host[(i, N)]
            Ks = [K1] + Ms[:-1]
            if kind == "reference":
                oracle.ref_chain(dt, B, As, N, Ms, Ks, threads=threads)
            else:
                oracle.chain(dt, B, As, N, Ms, Ks, mode=oracle.REF, threads=threads)
    one()
    times = []
    t_end = time.perf_counter() + budget_s
    while True:
        t0 = time.perf_counter()
        one()
        times.append(time.perf_counter() - t0)
        if steps is not None:
            if len(times) >= steps:
                break
        elif len(times) >= 3 and time.perf_counter() > t_end:
            break
    med = statistics.median(times)
    descr = {"kind": kind, "cores": threads, "cpu": model, "amx_available": amx,
             "amx_used": False,
             "sample": f"{len(reqs)} requests of the stream run one after another "
                       f"({fl / 1e9:.1f} GFLOP per step), median of {len(times)} steps"}
    return fl / med / 1e12, descr, times


def serve_cpu_inputs(sets, reqs, seed):
    rng = np.random.default_rng(seed)
    host = {}
    for i, N in reqs:
        dt, K1, Ms = sets[i]
        B, As, _ = make_inputs(dt, N, K1, Ms, int(rng.integers(1 << 30)))
        host[(i, N)] = (B, As)
    return host


def run_serve(args, world, rank, local_rank, ctx=None):
    """Serving loop at fractions of its measured capacity. g: the shared GPU
    context (None: the reference arm). Returns the line on rank 0, else None."""
    seed = 777
    sets = serve_sets(seed)
    nreq = args.serve_requests
    cpu_sample = serve_requests(seed + 5, sets, 24)
    config = {"workload": "serving stream: Poisson arrivals of chain requests, chain length "
                          "U{2..6}, dims log-uniform on multiples of 16 in [64, 4096], dtype mix "
                          "50% BF16 / 30% INT8 / 20% FP32 (3xTF32) over 64 resident weight sets; "
                          "activations and results resident in HBM",
              "requests_per_rate": nreq, "weight_sets": len(sets),
              "server": {"max_batch": 64, "slots": 2, "max_wait_us": 200,
                         "max_queue_us": f"{args.serve_deadline_us} at offered rates above "
                                         "capacity; 0 (no shedding) at or below it and for "
                                         "the capacity bursts"},
              "l2": "inputs of the stream far exceed L2; no flush between requests",
              "parallelism": f"dp{world} (each rank serves its own stream)"}
    metric = "served chain requests TFLOP/s (p50/p99 latency beside)"
    if args.impl == "reference":
        if rank != 0:
            return 0
        host = serve_cpu_inputs(sets, cpu_sample, seed + 6)
        tf, descr, times = serve_cpu(sets, cpu_sample, host, steps=args.steps)
        return {"impl": "reference", "metric": metric, "value": tf, "unit": "TFLOP/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * statistics.median(times), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "bf16/int8/f32 mix",
                "data": "synthetic (seeded)", "config": config,
                "cpu_baseline": dict(descr, value=tf, unit="TFLOP/s"),
                "e2e": {"value": tf, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}

    torch, fg, dist, dev = ctx.torch, ctx.fg, ctx.dist, ctx.dev
    fg.set_semantics("ref")
    fg.set_f32_algo("3xtf32")
    tdt = {"bf16": torch.bfloat16, "int8": torch.int8, "f32": torch.float32}
    W, Bs, Cs = [], [], []
    t_gen = time.perf_counter()
    for j, (dt, K1, Ms) in enumerate(sets):
        g = torch.Generator(device=dev).manual_seed(seed + j + 1000 * rank)
        Ks = [K1] + Ms[:-1]
        ws = []
        for m, k in zip(Ms, Ks):
            if dt == "int8":
                a = torch.randint(-127, 128, (m, k), generator=g, device=dev, dtype=torch.int8)
            else:
                a = (torch.randn(m, k, generator=g, device=dev) / float(np.sqrt(k))).to(tdt[dt])
                if dt == "bf16":
                    a = a.view(torch.int16)
            ws.append(fg.Weights(dt, a))
            del a
        W.append(ws)
        if dt == "int8":
            b = torch.randint(-127, 128, (K1 * 4096,), generator=g, device=dev, dtype=torch.int8)
        else:
            b = torch.randn(K1 * 4096, generator=g, device=dev).to(tdt[dt])
            if dt == "bf16":
                b = b.view(torch.int16)
        Bs.append(b)
        Cs.append([torch.empty(Ms[-1] * 4096, dtype=torch.int32 if dt == "int8" else torch.float32,
                               device=dev) for _ in range(4)])
    torch.cuda.synchronize(dev)
    t_gen = time.perf_counter() - t_gen
    weight_bytes = sum(w.nbytes for ws in W for w in ws)
    ring = [0] * len(sets)

    def materialise(reqs):
        out = []
        for i, N in reqs:
            dt, K1, Ms = sets[i]
            c = Cs[i][ring[i] % 4]
            ring[i] += 1
            out.append((dt, W[i], Bs[i][:K1 * N].view(K1, N), c[:Ms[-1] * N].view(Ms[-1], N)))
        return out

    # capacity and the points at or below it on a server that never sheds (a burst
    # queues every request at once, far past any deadline); the overload points on
    # one that sheds requests still queued args.serve_deadline_us after submit
    plain_srv = fg.Server(max_batch=64, slots=2, max_wait_us=200)
    shed_srv = None
    if args.serve_deadline_us > 0 and any(f > 1.0 for f in args.serve_rates):
        shed_srv = fg.Server(max_batch=64, slots=2, max_wait_us=200,
                             max_queue_us=args.serve_deadline_us)
    srv = plain_srv

    def run_point(reqs, at_us, prof=False):
        if dist:
            dist.barrier()
        fl = serve_flops(sets, reqs)
        mats = materialise(reqs)
        srv.reset_stats()
        l0 = fg.kernel_launches()
        if prof:
            fg.profile_begin()
        ids = srv.replay(mats, at_us)
        srv.drain()
        st = srv.stats()
        kernels = None
        if prof:
            torch.cuda.synchronize(dev)
            kernels = {name: fg.profile_query(k) for name, k in
                       (("bf16", fg.FG_PK_TC_BF16), ("int8", fg.FG_PK_TC_I8),
                        ("tf32x3", fg.FG_PK_TC_TF32X3))}
            fg.profile_end()
        launches = fg.kernel_launches() - l0
        for rid in ids:
            srv.wait(rid, shed_ok=True)
        return st, launches, kernels, sum(fl)

    # warm-up (memory pool at full batch size, tensor-map encoder, code paths), then
    # capacity: the better of two bursts (the loop's host side shares the CPU)
    warm = serve_requests(seed + 1, sets, min(2000, nreq))
    run_point(warm, [0.0] * len(warm))
    if shed_srv is not None:  # the same warm-up for the server of the overload points
        srv = shed_srv
        run_point(warm, [0.0] * len(warm))
        srv = plain_srv
    capacity = 0.0
    for k in range(2):
        burst = serve_requests(seed + 2 + 100 * k, sets, min(4000, nreq))
        st, _, _, fl = run_point(burst, [0.0] * len(burst))
        capacity = max(capacity, st["completed"] / st["span_s"])
    points = []
    sampler = ClockSampler(torch.cuda.current_device())
    launches_total = 0
    kernels = None
    rng = np.random.default_rng(seed + 3)
    with sampler:
        for k, frac in enumerate(args.serve_rates):
            if frac > 1.0 and shed_srv is not None:
                srv = shed_srv
            else:
                srv = plain_srv
            rate = frac * capacity
            reqs = serve_requests(seed + 10 + k, sets, nreq)
            at = np.cumsum(rng.exponential(1e6 / rate, size=nreq))
            under = [f for f in args.serve_rates if f <= 1.0] or args.serve_rates
            prof = frac == max(under)  # kernel times at the headline point
            st, launches, kern, fl = run_point(reqs, at.tolist(), prof=prof)
            launches_total += launches
            if prof:
                kernels = kern
            points.append({"offered_req_s": rate, "offered_frac_of_capacity": frac,
                           "served_req_s": st["completed"] / st["span_s"],
                           "tflops": st["flops"] / st["span_s"] / 1e12,
                           "p50_us": st["p50_us"], "p99_us": st["p99_us"],
                           "mean_us": st["mean_us"], "max_us": st["max_us"],
                           "batches": st["batches"], "mean_batch": st["mean_batch"],
                           "failed": st["failed"], "shed": st["shed"],
                           "shed_frac": st["shed"] / max(1, st["submitted"]),
                           "peak_bytes": st["peak_bytes"]})

    # end to end: host (pinned) activations in and results out inside each request
    e2e_n = min(nreq, 4000)
    reqs = serve_requests(seed + 50, sets, e2e_n)
    hB = [torch.empty(b.numel(), dtype=b.dtype, pin_memory=True) for b in Bs]
    for h, b in zip(hB, Bs):
        h.copy_(b)
    hC = [torch.empty(Cs[i][0].numel(), dtype=Cs[i][0].dtype, pin_memory=True)
          for i in range(len(sets))]
    mats, h2d, d2h = [], 0, 0
    for i, N in reqs:
        dt, K1, Ms = sets[i]
        b = hB[i][:K1 * N].view(K1, N).numpy()
        c = hC[i][:Ms[-1] * N].view(Ms[-1], N).numpy()
        mats.append((dt, W[i], b, c))
        h2d += b.nbytes
        d2h += c.nbytes
    rate = 0.6 * capacity
    at = np.cumsum(rng.exponential(1e6 / rate, size=e2e_n))
    srv = plain_srv
    srv.reset_stats()
    ids = srv.replay(mats, at.tolist())
    srv.drain()
    st_e2e = srv.stats()
    for rid in ids:
        srv.wait(rid, shed_ok=True)
    plain_srv.close()
    if shed_srv is not None:
        shed_srv.close()
    for ws in W:
        for w in ws:
            w.release()
    # the headline point: the highest offered rate at or below the measured capacity
    # (points above it show the shedding that keeps served latency bounded)
    sustained = [p for p in points if p["offered_frac_of_capacity"] <= 1.0] or points
    top = max(sustained, key=lambda p: p["offered_frac_of_capacity"])
    # whole job: throughput summed over the ranks' streams, latency the worst rank's
    job_tflops = top["tflops"]
    job_e2e = st_e2e["flops"] / st_e2e["span_s"] / 1e12
    lat = [top["p50_us"], top["p99_us"]]
    if dist:
        t = torch.tensor([job_tflops, job_e2e], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        job_tflops, job_e2e = float(t[0].item()), float(t[1].item())
        t = torch.tensor(lat, dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        lat = [float(x) for x in t.tolist()]
        dist.barrier()
    if rank != 0:
        return None

    peaks, peak_src = load_peaks()
    main = max(kernels.items(), key=lambda kv: kv[1][0]) if kernels else None
    roofline = None
    if main and main[1][0] > 0:
        name, (k_ms, k_n, k_fl) = main
        peak = {"bf16": peaks["bf16_tflops"], "int8": 2 * peaks["bf16_tflops"],
                "tf32x3": peaks["bf16_tflops"] / 6.0}[name]
        ach = k_fl / (k_ms / 1e3) / 1e12
        roofline = {"bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                    "frac": ach / peak, "traffic": None,
                    "kernel": f"grouped {name} kernel (the class with the most device time)",
                    "launches_timed": k_n, "avg_launch_us": 1e3 * k_ms / k_n,
                    "peak_source": ("bf16_tflops" if name == "bf16" else
                                    "2 x bf16_tflops" if name == "int8" else
                                    "bf16_tflops / 2 / 3") + f"; {peak_src}"}
    line = {"metric": metric, "value": job_tflops, "unit": "TFLOP/s", "n_gpus": world,
            "steps": len(points), "warmup": 1, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16/int8/f32(3xTF32) mix",
            "data": "synthetic (seeded; no dataset involved)", "config": config,
            "clocks": sampler.summary(), "gpu_launches": launches_total,
            "latency": {"p50_us": lat[0], "p99_us": lat[1], "ranks": "worst rank",
                        "at_offered_frac_of_capacity": top["offered_frac_of_capacity"]},
            "capacity_req_s": capacity, "points": points,
            "e2e": {"value": job_e2e, "unit": "TFLOP/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "step": f"{e2e_n} requests at 0.6 x capacity",
                    "p50_us": st_e2e["p50_us"], "p99_us": st_e2e["p99_us"],
                    "api": "fg_server_* with pinned host activations and results"},
            "roofline": roofline,
            "kernels": {k: {"ms": v[0], "launches": v[1],
                            "tflops": v[2] / (v[0] / 1e3) / 1e12 if v[0] else None}
                        for k, v in (kernels or {}).items()},
            "resident": {"weight_bytes": weight_bytes, "setup_s": t_gen}}
    if world == 1:
        host = serve_cpu_inputs(sets, cpu_sample, seed + 6)
        tf, descr, _ = serve_cpu(sets, cpu_sample, host, budget_s=args.cpu_budget)
        line["cpu_baseline"] = dict(descr, value=tf, unit="TFLOP/s")
    return line


class GpuCtx:
    """What every workload of our arm shares: torch, the library, the process
    group (N > 1), this rank's device and the L2-flush buffer."""

    def __init__(self, world, rank, local_rank):
        import torch
        import flashgemm_b200 as fg
        self.torch, self.fg = torch, fg
        self.world, self.rank, self.local_rank = world, rank, local_rank
        torch.cuda.set_device(local_rank)
        self.dev = torch.device("cuda", local_rank)
        self.dist = None
        if world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=self.dev)
            self.dist = dist
        fg.lib()
        fg.set_semantics("ref")
        fg.flashgemm_set_thread_num(1)
        # written between timed steps (outside their events): larger than the 126 MB L2
        self.flush = torch.empty(256 << 20, dtype=torch.uint8, device=self.dev)

    def max_over_ranks(self, *vals):
        if not self.dist:
            return vals
        t = self.torch.tensor(list(vals), dtype=self.torch.float64, device=self.dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return tuple(float(x) for x in t.tolist())

    def close(self):
        if self.dist:
            self.dist.barrier()
            self.dist.destroy_process_group()


# The reference's own three-stage chain table (multigemm/test/test_bf16_3.c:14-48; the
# FP32 and INT8 tests use the same shapes): N, K_1, (M_1, M_2, M_3)
REF_CHAINS = [
    (65536, 288, (32, 24, 144)), (16384, 1296, (144, 32, 192)), (16384, 1728, (192, 32, 192)),
    (4096, 4800, (192, 56, 336)), (4096, 8400, (336, 56, 336)), (50176, 288, (32, 16, 96)),
    (12544, 864, (96, 24, 144)), (12544, 1296, (144, 24, 144)), (3136, 1296, (144, 32, 192)),
    (3136, 1728, (192, 32, 192)),
]


def run_ref_table(g, reps=10):
    """Device time of every chain of the reference's table, BF16 and INT8, on the
    library's default path (narrow chains where measured faster), with narrow
    chains off (the fused chain kernel) and per GEMM. L2 flushed before every
    timed call, outside its events; seeded synthetic operands of the table's
    shapes."""
    torch, fg = g.torch, g.fg
    gen = torch.Generator(device=g.dev)
    gen.manual_seed(11)
    out = {"workload": "the reference's 10 three-stage chains (multigemm/test/test_bf16_3.c:14-48), "
                       "one call each, L2 flushed between calls",
           "l2": "flushed before every timed call (256 MiB write outside the events)"}
    launches0 = fg.kernel_launches()
    for dt in ("bf16", "int8"):
        rows, tot = [], {"default": 0.0, "narrow_off": 0.0, "per_gemm": 0.0}
        flops_all = bytes_all = 0.0
        for N, K1, Ms in REF_CHAINS:
            Ms = list(Ms)
            Ks = [K1] + Ms[:-1]
            if dt == "bf16":
                tB = torch.randn(K1, N, device=g.dev, generator=gen).to(torch.bfloat16).view(torch.int16)
                tA = [torch.randn(m, k, device=g.dev, generator=gen).div(k ** 0.5)
                      .to(torch.bfloat16).view(torch.int16) for m, k in zip(Ms, Ks)]
            else:
                tB = torch.randint(-3, 4, (K1, N), device=g.dev, generator=gen).to(torch.int8)
                tA = [torch.randint(0, 4, (m, k), device=g.dev, generator=gen).to(torch.int8)
                      for m, k in zip(Ms, Ks)]
            tC = torch.empty((Ms[-1], N), dtype=torch.int32 if dt == "int8" else torch.float32,
                             device=g.dev)
            row = {"N": N, "K1": K1, "M": Ms}
            for path in ("default", "narrow_off", "per_gemm"):
                fg.set_narrow("off" if path == "narrow_off" else "auto")
                fg.set_chain_mode("per_gemm" if path == "per_gemm" else "fused")
                try:
                    for _ in range(3):
                        fg.chain_dev(dt, tC, tB, N, tA, Ms, Ks)
                    torch.cuda.synchronize(g.dev)
                    ts = []
                    for i in range(reps):
                        g.flush.fill_(i & 0xFF)
                        a = torch.cuda.Event(enable_timing=True)
                        b = torch.cuda.Event(enable_timing=True)
                        a.record()
                        fg.chain_dev(dt, tC, tB, N, tA, Ms, Ks)
                        b.record()
                        torch.cuda.synchronize(g.dev)
                        ts.append(a.elapsed_time(b) * 1e3)
                    fg.sync()
                finally:
                    fg.set_narrow("auto")
                    fg.set_chain_mode("fused")
                us = sorted(ts)[reps // 2]
                row[f"us_{path}"] = round(us, 2)
                tot[path] += us
            fl = sum(2.0 * N * m * k for m, k in zip(Ms, Ks))
            elt = 2 if dt == "bf16" else 1
            by = K1 * N * elt + Ms[-1] * N * 4 + sum(m * k * elt for m, k in zip(Ms, Ks))
            flops_all += fl
            bytes_all += by
            rows.append(row)
        out[dt] = {
            "chains": rows,
            "total_us": {k: round(v, 1) for k, v in tot.items()},
            "tflops_default": flops_all / (tot["default"] * 1e-6) / 1e12,
            "gbs_default": bytes_all / (tot["default"] * 1e-6) / 1e9,
            "default_vs_narrow_off": tot["narrow_off"] / tot["default"],
            "default_vs_per_gemm": tot["per_gemm"] / tot["default"],
        }
    out["gpu_launches"] = fg.kernel_launches() - launches0
    return out


def measure_peaks(g, iters=20):
    """cuBLAS bursts at 8192^3 on this device in this run (torch): BF16, INT8
    (torch._int_mm), TF32 and plain FP32 (TF32 off) - the denominators of the
    dtypes the peaks file does not measure."""
    torch = g.torch
    n = 8192
    out = {}
    a16 = torch.randn(n, n, device=g.dev).to(torch.bfloat16)
    a8 = torch.randint(-127, 128, (n, n), device=g.dev, dtype=torch.int8)
    a32 = torch.randn(n, n, device=g.dev)
    prev = torch.backends.cuda.matmul.allow_tf32

    def burst(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize(g.dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(iters):
            fn()
        e1.record()
        torch.cuda.synchronize(g.dev)
        return 2.0 * n ** 3 * iters / (e0.elapsed_time(e1) / 1e3) / 1e12

    try:
        out["bf16_tflops"] = burst(lambda: a16 @ a16)
        out["int8_tops"] = burst(lambda: torch._int_mm(a8, a8))
        torch.backends.cuda.matmul.allow_tf32 = True
        out["tf32_tflops"] = burst(lambda: a32 @ a32)
        torch.backends.cuda.matmul.allow_tf32 = False
        out["fp32_tflops"] = burst(lambda: a32 @ a32)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    del a16, a8, a32
    torch.cuda.empty_cache()
    out["shape"] = "8192^3, cuBLAS through torch, 20-launch burst after 3 warm-up launches"
    return out


def pageable(a):
    """A copy of `a` in ordinary (pageable) host memory, as the reference's
    callers pass it (posix_memalign / malloc, multigemm/test/test_bf16_3.c:90-102)."""
    b = np.empty_like(a)
    b[...] = a
    return b


def run_chain_bench(args, g, workload, peaks_run=None):
    """One chain workload (or the FP32 SGEMM) on this rank: device-resident steps,
    the per-GEMM and cuBLAS comparators, end to end through the C ABI from pinned
    and from pageable host buffers, the roofline of the main kernel and the
    reference's CPU time. Returns the line on rank 0, else None."""
    torch, fg, dist, dev = g.torch, g.fg, g.dist, g.dev
    world, rank = g.world, g.rank
    dt, N_all, K1, Ms = WORKLOADS[workload]
    strong = args.scaling == "strong" and world > 1 and dt != "f32"
    if strong:
        # the ranks split one chain's columns (fg_split_columns), no collective
        c0, c1 = fg.shard_columns(N_all, world, rank)
        N = c1 - c0
    else:
        N = N_all
    metric = {"f32": "FP32 GEMM TFLOP/s"}.get(dt, "fused GEMM-chain TFLOP/s")
    config = {"workload": DESCR[workload], "dtype": dt, "N": N_all, "K1": K1, "M": Ms,
              "gflop_per_step_per_gpu": flops_of(N, K1, Ms) / 1e9,
              "semantics": "reference (panel permutation, INT8 tail rows)",
              "l2": "flushed between steps (256 MiB write outside the step events)",
              "parallelism": (f"dp{world} (one chain's {N_all} columns split across the ranks on "
                              "32-column panel boundaries, no collective)" if strong else
                              f"dp{world} (activation columns partitioned, no collective)")}

    # --------------------------------------------------------- device-resident step
    B, As, Ks = make_inputs(dt, N, K1, Ms, seed=1234 + rank)

    def to_dev(a):
        if a.dtype == np.uint16:
            a = a.view(np.int16)
        elif a.dtype == np.uint8:
            a = a.view(np.int8)
        return torch.from_numpy(a).to(dev)

    tB = to_dev(B)
    tA = [to_dev(a) for a in As]
    tC = torch.empty((Ms[-1], N), dtype=torch.int32 if dt == "int8" else torch.float32,
                     device=dev)
    flush = g.flush

    registered = None
    if dt == "f32":
        def step():
            fg.sgemm_dev(tC, tA[0], tB, Ms[0], N, K1, "ffma")
        kind = fg.FG_PK_FFMA
    elif dt == "int8":
        # weights resident as a server holds them: registered once (the reference's
        # INT8 tail rows prepared at registration); fg_chain_dev on unregistered
        # weights, which prepares them on every call, is timed beside it
        registered = [fg.Weights(dt, a) for a in tA]

        def step():
            fg.chain_registered(dt, tC, tB, N, registered)
        kind = fg.FG_PK_TC_I8
        config["weights"] = ("registered once (fg_weights_register: resident in HBM, INT8 tail "
                             "rows prepared at registration); value_unregistered: fg_chain_dev "
                             "preparing them on every call")
    else:
        def step():
            fg.chain_dev(dt, tC, tB, N, tA, Ms, Ks)
        kind = fg.FG_PK_TC_BF16

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize(dev)
    fg.sync()

    def timed(fn, sampler=None, prof=False):
        """Exactly args.steps steps, each bracketed by CUDA events on torch's
        stream (the library runs on that stream), L2 flushed between steps
        outside the events. Returns (sum of step ms, wall s, our launches,
        profile of the main kernel class)."""
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        stops = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
        l0 = fg.kernel_launches()
        if prof:
            fg.profile_begin()
        with (sampler if sampler is not None else _Null()):
            t_wall = time.perf_counter()
            for i in range(args.steps):
                flush.fill_(i & 0xFF)
                starts[i].record()
                fn()
                stops[i].record()
            torch.cuda.synchronize(dev)
            fg.sync()
            t_wall = time.perf_counter() - t_wall
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
        kp = None
        if prof:
            fg.profile_end()
            kp = fg.profile_query(kind)
        return (sum(s.elapsed_time(e) for s, e in zip(starts, stops)), t_wall,
                fg.kernel_launches() - l0, kp)

    # the step time without per-launch events (an event pair around every kernel
    # costs about 7 us of a 70 us BF16 step); then the same steps again with them,
    # for the main kernel's per-launch duration (the roofline)
    sampler = ClockSampler(torch.cuda.current_device())
    total_ms, t_wall, launches, _ = timed(step, sampler)
    _, _, _, (k_ms, k_n, k_fl) = timed(step, prof=True)

    unreg = None
    if registered is not None:
        def step_unreg():
            fg.chain_dev(dt, tC, tB, N, tA, Ms, Ks)
        for _ in range(max(args.warmup, 3)):
            step_unreg()
        unreg, _, _, _ = timed(step_unreg)

    # the same steps through the plain per-GEMM path (one launch per GEMM)
    per_gemm = None
    if dt != "f32":
        fg.set_chain_mode("per_gemm")
        for _ in range(max(args.warmup, 3)):
            step()
        pg_ms, _, pg_launches, _ = timed(step)
        fg.set_chain_mode("fused")
        per_gemm = (pg_ms, pg_launches)

    # a plain library path beside it: one cuBLAS GEMM per stage (torch), the
    # narrowing between stages as separate kernels, intermediates in HBM (same
    # shapes and dtypes; INT8 with signed weights, cuBLAS having no unsigned x
    # signed GEMM; no panel permutation). FP32: cuBLAS SGEMM with TF32 off.
    if dt == "bf16":
        cA = [a.view(torch.bfloat16) for a in tA]
        cB = tB.view(torch.bfloat16)

        def plain():
            x = cB
            for a in cA:
                x = a @ x  # FP32 accumulation, BF16 result (RNE)
            return x.float()
    elif dt == "int8":
        def plain():
            x = tB
            for i, a in enumerate(tA):
                y = torch._int_mm(a, x)
                x = y if i == len(tA) - 1 else y.clamp_(-128, 127).to(torch.int8)
            return x
    else:
        def plain():
            return torch.matmul(tA[0], tB, out=tC)
    prev_tf32 = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        for _ in range(max(args.warmup, 3)):
            plain()
        cublas, _, _, _ = timed(plain)
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev_tf32

    total_ms, = g.max_over_ranks(total_ms)
    if per_gemm:
        per_gemm = (g.max_over_ranks(per_gemm[0])[0], per_gemm[1])
    cublas, = g.max_over_ranks(cublas)
    if unreg is not None:
        unreg, = g.max_over_ranks(unreg)
    step_flops = flops_of(N, K1, Ms)
    # whole-job work per step: every rank's columns (weak: N each; strong: one chain)
    job_flops = flops_of(N_all, K1, Ms) if strong else world * step_flops
    value = job_flops * args.steps / (total_ms / 1e3) / 1e12

    # --------------------------------------------------------- end to end through the C ABI
    e2e_steps = args.e2e_steps or min(args.steps, 200)

    def e2e_run(hB, hA, hC):
        trip = []
        for a, m, k in zip(hA, Ms, Ks):
            trip += [a, m, k]
        if dt == "f32":
            def one():
                fg.LibShalom_sgemm_mp(0, 0, hC, hA[0], hB, Ms[0], N, K1, check=True)
        else:
            fn = {"bf16": fg.flashgemm_multi_bf16bf16f32,
                  "int8": fg.flashgemm_multi_int8uint8int32}[dt]

            def one():
                fn(hC, hB, N, len(Ms), *trip, check=True)
        for _ in range(3):
            one()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            one()
        sec, = g.max_over_ranks(time.perf_counter() - t0)
        return job_flops * e2e_steps / sec / 1e12

    pin = lambda a: torch.from_numpy(a).pin_memory().numpy()  # noqa: E731
    out_np = np.int32 if dt == "int8" else np.float32
    hB, hA, hC = pin(B), [pin(a) for a in As], pin(np.zeros((Ms[-1], N), out_np))
    e2e_value = e2e_run(hB, hA, hC)
    pB, pA, pC = pageable(B), [pageable(a) for a in As], np.zeros((Ms[-1], N), out_np)
    e2e_pageable = e2e_run(pB, pA, pC)
    h2d = hB.nbytes + sum(a.nbytes for a in hA)
    d2h = hC.nbytes
    del hB, hA, hC, pB, pA, pC

    if registered is not None:
        for w in registered:
            w.release()
    if rank != 0:
        return None
    peaks, peak_src = load_peaks()
    peaks_run = peaks_run or {}
    achieved = k_fl / (k_ms / 1e3) / 1e12 if k_ms > 0 else None
    if dt == "bf16":
        peak, peak_name = peaks.get("bf16_tflops"), "bf16_tflops (cuBLAS BF16 burst)"
        peak_src_s = peak_src
    elif dt == "int8":
        if peaks_run.get("int8_tops"):
            peak = peaks_run["int8_tops"]
            peak_name = "cuBLAS INT8 burst at 8192^3 (torch._int_mm), measured in this run"
            peak_src_s = "measured"
        else:
            peak = 2 * peaks.get("bf16_tflops")
            peak_name = "2 x bf16_tflops (INT8 = 2x BF16 per clock)"
            peak_src_s = peak_src
    else:
        sm_mhz = peaks.get("sm_max_mhz", 1965.0)
        peak = 148 * 256 * sm_mhz * 1e6 / 1e12
        peak_name = "148 SMs x 128 FFMA/clk x 2 x sm_max_mhz (datasheet-style FFMA peak)"
        peak_src_s = "datasheet arithmetic"
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            traffic = json.load(f).get(workload)
    except (OSError, ValueError):
        traffic = None
    roofline = {"bound": "tensor" if dt != "f32" else "ffma", "achieved": achieved,
                "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if achieved and peak else None,
                "traffic": traffic.get("bytes_per_launch") if traffic else None,
                "kernel": ("fg::tc_chain_kernel (whole chain, one launch)" if dt != "f32"
                           else "fg::ffma_sgemm_kernel"),
                "launches_timed": k_n, "avg_launch_us": 1e3 * k_ms / k_n if k_n else None,
                "launch_timing": "CUDA events around every launch of the main kernel, on its "
                                 "stream, in a second timed pass of the same steps (the step "
                                 "times come from a pass without them)",
                "peak_source": f"{peak_name}; {peak_src_s}"}
    if dt == "int8":
        roofline["frac_of_2x_bf16"] = achieved / (2 * peaks.get("bf16_tflops")) if achieved else None
    if dt == "f32" and peaks_run.get("fp32_tflops"):
        roofline["frac_of_cublas_fp32_burst"] = achieved / peaks_run["fp32_tflops"] if achieved else None

    line = {"metric": metric, "value": value, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "strong" if strong else "weak",
            "vs_baseline": None, "dtype": dt,
            "data": "synthetic (seeded; no dataset involved)", "config": config,
            "clocks": sampler.summary(), "gpu_launches": launches,
            "e2e": {"value": e2e_value, "unit": "TFLOP/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                    "api": "flashgemm_multi_*/LibShalom_sgemm_mp, pinned host buffers",
                    "pageable_value": e2e_pageable,
                    "pageable_api": "the same calls on ordinary (pageable) host buffers"},
            "roofline": roofline, "wall_s_timed_region": t_wall}
    if unreg is not None:
        line["value_unregistered"] = job_flops * args.steps / (unreg / 1e3) / 1e12
        line["ms_per_step_unregistered"] = unreg / args.steps
    if per_gemm:
        pg_value = job_flops * args.steps / (per_gemm[0] / 1e3) / 1e12
        line["per_gemm"] = {"value": pg_value, "unit": "TFLOP/s",
                            "ms_per_step": per_gemm[0] / args.steps,
                            "launches": per_gemm[1],
                            "path": "one tensor-core launch per GEMM (FG_CHAIN_PER_GEMM)"}
        line["fused_vs_per_gemm"] = value / pg_value
    cb_value = job_flops * args.steps / (cublas / 1e3) / 1e12
    if dt == "f32":
        line["cublas_sgemm"] = {"value": cb_value, "unit": "TFLOP/s",
                                "ms_per_step": cublas / args.steps,
                                "path": "torch.matmul FP32 (cuBLAS SGEMM, TF32 off), same operands"}
        line["ffma_vs_cublas_sgemm"] = value / cb_value
    else:
        line["cublas_per_gemm"] = {
            "value": cb_value, "unit": "TFLOP/s", "ms_per_step": cublas / args.steps,
            "path": "torch.matmul / torch._int_mm (cuBLAS) per GEMM, narrowing as separate "
                    "kernels, intermediates in HBM; INT8 with signed weights, no panel permutation"}
        line["fused_vs_cublas_per_gemm"] = value / cb_value
    if world == 1:
        tf, descr, _ = time_cpu(workload, budget_s=args.cpu_budget)
        line["cpu_baseline"] = dict(descr, value=tf, unit="TFLOP/s")
    return line


def reference_line(args, workload):
    """--impl reference for a chain / SGEMM workload: the reference's own CPU
    implementation on all host threads, on a bounded column sample."""
    dt, N, K1, Ms = WORKLOADS[workload]
    metric = {"f32": "FP32 GEMM TFLOP/s"}.get(dt, "fused GEMM-chain TFLOP/s")
    config = {"workload": DESCR[workload], "dtype": dt, "N": N, "K1": K1, "M": Ms,
              "gflop_per_step_per_gpu": flops_of(N, K1, Ms) / 1e9,
              "semantics": "reference (panel permutation, INT8 tail rows)",
              "l2": "flushed between steps (256 MiB write outside the step events)",
              "parallelism": f"dp{args.gpus} (activation columns partitioned, no collective)"}
    tf, descr, times = time_cpu(workload, steps=args.steps, warmup=args.warmup)
    return {"impl": "reference", "metric": metric, "value": tf, "unit": "TFLOP/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * statistics.median(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dt,
            "data": "synthetic (seeded)", "config": config,
            "cpu_baseline": dict(descr, value=tf, unit="TFLOP/s"),
            "e2e": {"value": tf, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


# keys of a sub-object: the workload's own figures, without the top-level
# contract fields it shares with the headline line
_SUB_DROP = ("n_gpus", "warmup", "higher_is_better", "scaling", "vs_baseline", "data")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 200; f32-groups 20)")
    ap.add_argument("--warmup", type=int, default=None,
                    help="untimed steps (default 10; f32-groups 3)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="all",
                    choices=["all"] + list(WORKLOADS) + ["f32-groups", "serve", "ref-chains"],
                    help="all (default): the BF16 chain as the headline line, with the INT8 "
                         "chain, the FP32 SGEMM, a grouped FP32 subset and a serving point as "
                         "sub-objects of the same line")
    ap.add_argument("--group-chains", type=int, default=None,
                    help="f32-groups: chains in the group (default 512; 128 within 'all')")
    ap.add_argument("--skinny-only", action="store_true",
                    help="f32-groups: only the tall-skinny chains (a small HBM-bound profiling case)")
    ap.add_argument("--serve-requests", type=int, default=None,
                    help="serve: Poisson requests per rate point (default 20000; 4000 within 'all')")
    ap.add_argument("--serve-rates", type=float, nargs="+", default=None,
                    help="serve: offered rates as fractions of the measured capacity "
                         "(default 0.3 0.6 0.9; 0.6 within 'all')")
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"],
                    help="N > 1, chain workloads: weak (every rank its own full chain) or "
                         "strong (the ranks split one chain's columns)")
    ap.add_argument("--serve-deadline-us", type=int, default=20000,
                    help="serve: the server sheds requests still queued this long after submit")
    ap.add_argument("--e2e-steps", type=int, default=None,
                    help="steps of the host-buffer C-ABI measurement (default: min(steps, 200))")
    ap.add_argument("--cpu-budget", type=float, default=None,
                    help="seconds of reference CPU work for each cpu_baseline leg "
                         "(default 12; 6 within 'all')")
    args = ap.parse_args()
    combined = args.workload == "all"
    grouped = args.workload == "f32-groups"
    if args.steps is None:
        args.steps = 20 if grouped else 200
    if args.warmup is None:
        args.warmup = 3 if grouped else 10
    if args.group_chains is None:
        args.group_chains = 128 if combined else GROUP_CHAINS
    if args.serve_requests is None:
        args.serve_requests = 4000 if combined else 20000
    if args.serve_rates is None:
        args.serve_rates = [0.6, 1.2] if combined else [0.3, 0.6, 0.9, 1.2]
    if args.cpu_budget is None:
        args.cpu_budget = 6.0 if combined else 12.0

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        # rank 0 alone times the reference's CPU implementation; the others exit
        if rank != 0:
            return 0
        if grouped:
            line = run_groups(args, world, rank, local_rank)
        elif args.workload == "serve":
            line = run_serve(args, world, rank, local_rank)
        elif args.workload == "ref-chains":
            line = {"impl": "reference", "unavailable": "the chain table is a sub-object of the "
                    "default line; its reference CPU timing is the chain workloads' cpu_baseline"}
        else:
            line = reference_line(args, "bf16-chain" if combined else args.workload)
        print(json.dumps(line), flush=True)
        return 0

    g = GpuCtx(world, rank, local_rank)
    if grouped:
        line = run_groups(args, world, rank, local_rank, g)
    elif args.workload == "serve":
        line = run_serve(args, world, rank, local_rank, g)
    elif args.workload == "ref-chains":
        line = run_ref_table(g)
    elif not combined:
        line = run_chain_bench(args, g, args.workload)
    else:
        peaks_run = measure_peaks(g)
        line = run_chain_bench(args, g, "bf16-chain", peaks_run)
        subs = {}
        subs["int8_chain"] = run_chain_bench(args, g, "int8-chain", peaks_run)
        subs["f32_gemm"] = run_chain_bench(args, g, "f32-gemm", peaks_run)
        gargs = argparse.Namespace(**vars(args))
        gargs.steps, gargs.warmup = min(args.steps, 20), 3
        subs["f32_groups"] = run_groups(gargs, world, rank, local_rank, g)
        subs["serve"] = run_serve(args, world, rank, local_rank, g)
        subs["ref_chains"] = run_ref_table(g)
        if rank == 0:
            for k, v in subs.items():
                line[k] = {kk: vv for kk, vv in v.items() if kk not in _SUB_DROP}
            line["gpu_launches_all_workloads"] = line["gpu_launches"] + sum(
                v.get("gpu_launches") or 0 for v in subs.values())
            line["peaks_this_run"] = peaks_run
            grp = subs["f32_groups"]
            if grp.get("roofline") and peaks_run.get("tf32_tflops"):
                r = grp["roofline"]
                r["frac_of_measured_tf32_div3"] = r["achieved"] / (peaks_run["tf32_tflops"] / 3.0)
    g.close()
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
