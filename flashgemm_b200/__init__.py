"""flashgemm-b200: the reference flashgemm hot path (FP32 SGEMM and FP32 / BF16 /
INT8 GEMM chains) on B200 tensor cores, behind the reference's own C entry points.

This module is the Python-side mirror of that C ABI (ctypes over the in-tree
libflashgemm_b200.so). The functions named like the reference's take the
reference's arguments in the reference's order:

    flashgemm_set_thread_num(num)                               flashgemm.h:19
    flashgemm_multi_f32f32f32(C, B, N, num_gemm, A1, M1, K1, ...)      :21
    flashgemm_multi_bf16bf16f32(C, B, N, num_gemm, A1, M1, K1, ...)    :23
    flashgemm_multi_int8uint8int32(C, B, N, num_gemm, A1, M1, K1, ...) :25
    LibShalom_sgemm_mp(transa, transb, C, A, B, M, N, K)        FP32_ID23.c:35

with numpy arrays (host memory) for the matrices. Like the reference they
return nothing; pass check=True to raise FlashgemmError on a failed call. The
device-pointer entry points (chain_dev, sgemm_dev) take torch CUDA tensors.
There is no CPU fallback: without the library or a B200, calls fail loudly.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libflashgemm_b200.so")

FG_OK, FG_ERR_INVALID, FG_ERR_UNSUPPORTED, FG_ERR_CUDA, FG_ERR_NO_DEVICE, FG_ERR_TIMEOUT, \
    FG_ERR_NOMEM, FG_ERR_BUSY = range(8)
FG_SEM_REF, FG_SEM_MATH = 0, 1
FG_F32_FFMA, FG_F32_3XTF32 = 0, 1
FG_DT_F32, FG_DT_BF16, FG_DT_INT8 = 0, 1, 2
_DT = {"f32": FG_DT_F32, "bf16": FG_DT_BF16, "int8": FG_DT_INT8}

_P = ctypes.c_void_p
_L = ctypes.c_long
_lib = None


class FlashgemmError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"flashgemm-b200 status {status}: {msg}")
        self.status = status


def lib():
    """Load libflashgemm_b200.so (built by flashgemm_b200/build.py)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `python flashgemm_b200/build.py`")
        L = ctypes.CDLL(LIB_PATH)
        L.fg_last_error.restype = ctypes.c_char_p
        L.fg_version.restype = ctypes.c_char_p
        L.fg_kernel_launches.restype = ctypes.c_ulonglong
        for name in ("flashgemm_multi_f32f32f32", "flashgemm_multi_bf16bf16f32",
                     "flashgemm_multi_int8uint8int32"):
            f = getattr(L, name)
            f.restype = None
            f.argtypes = [_P, _P, _L, ctypes.c_int]  # then (ptr, long, long) triples
        L.LibShalom_sgemm_mp.restype = None
        L.LibShalom_sgemm_mp.argtypes = [ctypes.c_int, ctypes.c_int, _P, _P, _P, _L, _L, _L]
        L.Small_NGM_NN_SGEMM.argtypes = [_P, _P, _P, _L, _L, _L, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int]
        L.Small_MGN_NN_SGEMM.argtypes = L.Small_NGM_NN_SGEMM.argtypes
        L.fg_chain_dev.argtypes = [ctypes.c_int, _P, _P, _L, ctypes.c_int, _P, _P, _P, _P]
        L.fg_sgemm_dev.argtypes = [_P, _P, _P, _L, _L, _L, ctypes.c_int, _P]
        _lib = L
    return _lib


def last_status():
    return lib().fg_last_status()


def last_error():
    return lib().fg_last_error().decode()


def _check(check):
    st = lib().fg_last_status()
    if check and st != FG_OK:
        raise FlashgemmError(st, last_error())
    return st


def version():
    return lib().fg_version().decode()


def kernel_launches():
    return int(lib().fg_kernel_launches())


def set_semantics(sem):
    lib().fg_set_semantics({"ref": FG_SEM_REF, "math": FG_SEM_MATH}.get(sem, sem))


def get_semantics():
    return lib().fg_get_semantics()


def set_f32_algo(algo):
    lib().fg_set_f32_algo({"ffma": FG_F32_FFMA, "3xtf32": FG_F32_3XTF32}.get(algo, algo))


def set_sgemm_algo(algo):
    lib().fg_set_sgemm_algo({"ffma": FG_F32_FFMA, "3xtf32": FG_F32_3XTF32}.get(algo, algo))


FG_CHAIN_FUSED, FG_CHAIN_PER_GEMM = 0, 1


def set_chain_mode(mode):
    lib().fg_set_chain_mode({"fused": FG_CHAIN_FUSED, "per_gemm": FG_CHAIN_PER_GEMM}.get(mode, mode))


def get_chain_mode():
    return lib().fg_get_chain_mode()


FG_NARROW_OFF, FG_NARROW_ALWAYS, FG_NARROW_AUTO = 0, 1, 2


def set_narrow(mode):
    """When fused BF16 / INT8 chains keep narrow intermediates on chip:
    "auto" (where measured faster), "always" or "off" (fg_set_narrow)."""
    lib().fg_set_narrow({"off": FG_NARROW_OFF, "always": FG_NARROW_ALWAYS,
                         "auto": FG_NARROW_AUTO}.get(mode, mode))


def get_narrow():
    return {FG_NARROW_OFF: "off", FG_NARROW_ALWAYS: "always", FG_NARROW_AUTO: "auto"}[lib().fg_get_narrow()]


def sync():
    st = lib().fg_sync()
    if st != FG_OK:
        raise FlashgemmError(st, last_error())


def selftest_timeout(limit_us=2000):
    """Run the failure-detection self-test (fg_selftest_timeout): a fused chain
    whose second stage waits on a dependency nothing releases, its waits
    limited to limit_us. Returns the status the host read (FG_ERR_TIMEOUT when
    detection works); raises nothing."""
    return lib().fg_selftest_timeout(int(limit_us))


# ------------------------------------------------------------ reference entry points

def _host_ptr(a, dtype):
    if not isinstance(a, np.ndarray) or not a.flags["C_CONTIGUOUS"]:
        raise TypeError("expected a C-contiguous numpy array")
    if a.dtype != dtype:
        raise TypeError(f"expected {np.dtype(dtype)}, got {a.dtype}")
    return a.ctypes.data_as(_P)


def _triples(args, adtype):
    if len(args) % 3:
        raise TypeError("weights come as (A_i, M_i, K_i) triples")
    out = []
    for i in range(0, len(args), 3):
        A, M, K = args[i:i + 3]
        out += [_host_ptr(A, adtype), _L(int(M)), _L(int(K))]
    return out


def flashgemm_set_thread_num(num):
    lib().flashgemm_set_thread_num(int(num))


def flashgemm_thread_num():
    return ctypes.c_int.in_dll(lib(), "flashgemm_thread_num").value


def flashgemm_multi_f32f32f32(C, B, N, num_gemm, *triples, check=False):
    lib().flashgemm_multi_f32f32f32(_host_ptr(C, np.float32), _host_ptr(B, np.float32), int(N),
                                    int(num_gemm), *_triples(triples, np.float32))
    return _check(check)


def flashgemm_multi_bf16bf16f32(C, B, N, num_gemm, *triples, check=False):
    lib().flashgemm_multi_bf16bf16f32(_host_ptr(C, np.float32), _host_ptr(B, np.uint16), int(N),
                                      int(num_gemm), *_triples(triples, np.uint16))
    return _check(check)


def flashgemm_multi_int8uint8int32(C, B, N, num_gemm, *triples, check=False):
    lib().flashgemm_multi_int8uint8int32(_host_ptr(C, np.int32), _host_ptr(B, np.uint8), int(N),
                                         int(num_gemm), *_triples(triples, np.int8))
    return _check(check)


def LibShalom_sgemm_mp(transa, transb, C, A, B, M, N, K, check=False):
    lib().LibShalom_sgemm_mp(int(transa), int(transb), _host_ptr(C, np.float32),
                             _host_ptr(A, np.float32), _host_ptr(B, np.float32), int(M), int(N),
                             int(K))
    return _check(check)


def LibShalom_set_thread_nums(num):
    lib().LibShalom_set_thread_nums(int(num))


def Small_NGM_NN_SGEMM(C, A, B, M, N, K, NUM, Tm, Tn, check=False):
    lib().Small_NGM_NN_SGEMM(_host_ptr(C, np.float32), _host_ptr(A, np.float32),
                             _host_ptr(B, np.float32), int(M), int(N), int(K), NUM, Tm, Tn)
    return _check(check)


def Small_MGN_NN_SGEMM(C, A, B, M, N, K, NUM, Tm, Tn, check=False):
    lib().Small_MGN_NN_SGEMM(_host_ptr(C, np.float32), _host_ptr(A, np.float32),
                             _host_ptr(B, np.float32), int(M), int(N), int(K), NUM, Tm, Tn)
    return _check(check)


# ------------------------------------------------------------ device entry points

def chain_dev(dtype, C, B, N, As, Ms, Ks, stream=None):
    """Chain on torch CUDA tensors (contiguous). dtype: 'f32' | 'bf16' | 'int8'.
    stream: a torch.cuda.Stream (default: torch's current stream)."""
    import torch
    n = len(As)
    aptr = (_P * n)(*[a.data_ptr() for a in As])
    ms = (ctypes.c_long * n)(*[int(m) for m in Ms])
    ks = (ctypes.c_long * n)(*[int(k) for k in Ks])
    s = (stream or torch.cuda.current_stream()).cuda_stream
    st = lib().fg_chain_dev(_DT[dtype], C.data_ptr(), B.data_ptr(), int(N), n, aptr, ms, ks, s)
    if st != FG_OK:
        raise FlashgemmError(st, last_error())


def sgemm_dev(C, A, B, M, N, K, algo="ffma", stream=None):
    import torch
    a = {"ffma": FG_F32_FFMA, "3xtf32": FG_F32_3XTF32}[algo]
    s = (stream or torch.cuda.current_stream()).cuda_stream
    st = lib().fg_sgemm_dev(C.data_ptr(), A.data_ptr(), B.data_ptr(), int(M), int(N), int(K), a, s)
    if st != FG_OK:
        raise FlashgemmError(st, last_error())


# ------------------------------------------------------------ per-launch timing

FG_PK_TC_BF16, FG_PK_TC_I8, FG_PK_TC_TF32X3, FG_PK_FFMA, FG_PK_AUX = range(5)


def profile_begin():
    st = lib().fg_profile_begin()
    if st != FG_OK:
        raise FlashgemmError(st, last_error())


def profile_end():
    lib().fg_profile_end()


def profile_query(kind=-1):
    """(device ms, launches, algorithmic FLOPs) of the kernels of one class
    launched since profile_begin(); kind=-1 sums every class."""
    ms = ctypes.c_double()
    n = ctypes.c_ulonglong()
    fl = ctypes.c_double()
    st = lib().fg_profile_query(int(kind), ctypes.byref(ms), ctypes.byref(n), ctypes.byref(fl))
    if st != FG_OK:
        raise FlashgemmError(st, last_error())
    return ms.value, int(n.value), fl.value


# ------------------------------------------------------------ multi-GPU partitioning

def shard_columns(N, world, rank):
    """Column range [start, stop) of the activations/outputs that `rank` of
    `world` owns when one chain is split across GPUs (the library's
    fg_split_columns; host arithmetic, no device needed). The chain is
    independent per column except that the reference's between-stage
    permutation mixes the columns of each 32-column panel, so shards are cut on
    panel boundaries: each rank then runs the unchanged chain on its slice of B
    and writes its slice of C, with no collective on the data path."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    L = lib()
    L.fg_split_columns.argtypes = [_L, ctypes.c_int, ctypes.c_int, _P, _P]
    c0, c1 = ctypes.c_long(), ctypes.c_long()
    st = L.fg_split_columns(int(N), int(world), int(rank), ctypes.byref(c0), ctypes.byref(c1))
    if st != FG_OK:
        raise FlashgemmError(st, last_error())
    return c0.value, c1.value


def chain_multi_device(dtype, C, B, N, As, Ms, Ks, devices):
    """One chain on host (numpy) operands split by columns across `devices`
    (fg_chain_multi_device): the reference entry points' semantics, bit for
    bit the single-device result."""
    L = lib()
    L.fg_chain_multi_device.argtypes = [ctypes.c_int, _P, _P, _L, ctypes.c_int, _P, _P, _P,
                                        ctypes.c_int, _P]
    n = len(As)
    adt = {"f32": np.float32, "bf16": np.uint16, "int8": np.int8}[dtype]
    bdt = {"f32": np.float32, "bf16": np.uint16, "int8": np.uint8}[dtype]
    odt = np.int32 if dtype == "int8" else np.float32
    aptr = (_P * n)(*[_host_ptr(a, adt) for a in As])
    ms = (ctypes.c_long * n)(*[int(m) for m in Ms])
    ks = (ctypes.c_long * n)(*[int(k) for k in Ks])
    dv = (ctypes.c_int * len(devices))(*[int(d) for d in devices])
    st = L.fg_chain_multi_device(_DT[dtype], _host_ptr(C, odt), _host_ptr(B, bdt), int(N), n, aptr,
                                 ms, ks, len(devices), dv)
    if st != FG_OK:
        raise FlashgemmError(st, last_error())


# ------------------------------------------------------------ weight registry

FG_MEM_HOST, FG_MEM_DEVICE = 0, 1


class Weights:
    """A weight matrix registered on the current device (fg_weights_register):
    copied once in the kernels' layout with its derived forms prepared once."""

    def __init__(self, dtype, A, M=None, K=None):
        L = lib()
        L.fg_weights_register.argtypes = [ctypes.c_int, _P, _L, _L, ctypes.c_int,
                                          ctypes.POINTER(_P)]
        L.fg_weights_bytes.restype = _L
        L.fg_weights_bytes.argtypes = [_P]
        L.fg_weights_release.argtypes = [_P]
        if isinstance(A, np.ndarray):
            M, K = A.shape if M is None else (M, K)
            ptr, where = A.ctypes.data_as(_P), FG_MEM_HOST
        else:  # torch CUDA tensor
            M, K = tuple(A.shape) if M is None else (M, K)
            ptr, where = _P(A.data_ptr()), FG_MEM_DEVICE
        h = _P()
        st = L.fg_weights_register(_DT[dtype], ptr, int(M), int(K), where, ctypes.byref(h))
        if st != FG_OK:
            raise FlashgemmError(st, last_error())
        self.handle, self.dtype, self.M, self.K = h, dtype, int(M), int(K)

    @property
    def nbytes(self):
        return int(lib().fg_weights_bytes(self.handle))

    def release(self):
        if self.handle:
            lib().fg_weights_release(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.release()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


def chain_registered(dtype, C, B, N, weights, stream=None):
    """Chain on registered weights (list of Weights) with device B and C."""
    import torch
    L = lib()
    L.fg_chain_registered.argtypes = [ctypes.c_int, _P, _P, _L, ctypes.c_int, _P, _P]
    n = len(weights)
    hs = (_P * n)(*[w.handle for w in weights])
    s = (stream or torch.cuda.current_stream()).cuda_stream
    st = L.fg_chain_registered(_DT[dtype], C.data_ptr(), B.data_ptr(), int(N), n, hs, s)
    if st != FG_OK:
        raise FlashgemmError(st, last_error())


class _ChainDesc(ctypes.Structure):
    _fields_ = [("C", _P), ("B", _P), ("N", _L), ("num_gemm", ctypes.c_int), ("W", _P)]


def _descs(chains):
    keep = []
    descs = (_ChainDesc * len(chains))()
    for d, (C, B, N, W) in zip(descs, chains):
        hs = (_P * len(W))(*[w.handle for w in W])
        keep.append(hs)
        d.C, d.B, d.N, d.num_gemm = C.data_ptr(), B.data_ptr(), int(N), len(W)
        d.W = ctypes.cast(hs, _P)
    return descs, keep


def chain_group(dtype, chains, stream=None):
    """Many chains in one grouped launch. chains: list of (C, B, N, [Weights])
    with torch CUDA tensors for C and B."""
    import torch
    L = lib()
    L.fg_chain_group.argtypes = [ctypes.c_int, ctypes.c_int, _P, _P]
    descs, keep = _descs(chains)
    s = (stream or torch.cuda.current_stream()).cuda_stream
    st = L.fg_chain_group(_DT[dtype], len(chains), ctypes.cast(descs, _P), s)
    if st != FG_OK:
        raise FlashgemmError(st, last_error())


FG_GROUP_AUTO, FG_GROUP_PAIR, FG_GROUP_SINGLE_256, FG_GROUP_SINGLE_128 = -1, 0, 1, 2
FG_ORDER_AUTO, FG_ORDER_FUSED, FG_ORDER_LEVELS = -1, 0, 1


def set_group_config(kernel=FG_GROUP_AUTO, order=FG_ORDER_AUTO):
    """Kernel (FG_GROUP_*) and stage order (FG_ORDER_*) of later grouped launches."""
    L = lib()
    L.fg_set_group_config.restype = None
    L.fg_set_group_config(int(kernel), int(order))


def get_group_config():
    L = lib()
    k, o = ctypes.c_int(), ctypes.c_int()
    L.fg_get_group_config.restype = None
    L.fg_get_group_config(ctypes.byref(k), ctypes.byref(o))
    return k.value, o.value


def group_choice(dtype, chains):
    """(kernel, order) a grouped launch of these chains would use now."""
    L = lib()
    descs, keep = _descs(chains)
    k, o = ctypes.c_int(), ctypes.c_int()
    L.fg_group_choice.argtypes = [ctypes.c_int, ctypes.c_int, _P, _P, _P]
    st = L.fg_group_choice(_DT[dtype], len(chains), ctypes.cast(descs, _P), ctypes.byref(k),
                           ctypes.byref(o))
    if st != FG_OK:
        raise FlashgemmError(st, last_error())
    return k.value, o.value


def autotune_group(dtype, chains, iters=3):
    """Time every kernel / order candidate on this group; returns (kernel, order, ms)
    and remembers the choice for groups of the same shapes."""
    L = lib()
    descs, keep = _descs(chains)
    k, o, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    L.fg_autotune_group.argtypes = [ctypes.c_int, ctypes.c_int, _P, ctypes.c_int, _P, _P, _P]
    st = L.fg_autotune_group(_DT[dtype], len(chains), ctypes.cast(descs, _P), int(iters),
                             ctypes.byref(k), ctypes.byref(o), ctypes.byref(ms))
    if st != FG_OK:
        raise FlashgemmError(st, last_error())
    return k.value, o.value, ms.value


def autotune_save(path):
    L = lib()
    L.fg_autotune_save.argtypes = [ctypes.c_char_p]
    if L.fg_autotune_save(str(path).encode()) != FG_OK:
        raise FlashgemmError(last_status(), last_error())


def autotune_load(path):
    L = lib()
    L.fg_autotune_load.argtypes = [ctypes.c_char_p]
    if L.fg_autotune_load(str(path).encode()) != FG_OK:
        raise FlashgemmError(last_status(), last_error())


class Plan:
    """A planned grouped launch bound to its chains' buffers (fg_plan_create)."""

    def __init__(self, dtype, chains):
        L = lib()
        descs, keep = _descs(chains)
        h = _P()
        L.fg_plan_create.argtypes = [ctypes.c_int, ctypes.c_int, _P, _P]
        st = L.fg_plan_create(_DT[dtype], len(chains), ctypes.cast(descs, _P), ctypes.byref(h))
        if st != FG_OK:
            raise FlashgemmError(st, last_error())
        self.handle = h.value
        self._chains = chains  # the plan points at these tensors

    def launch(self, stream=None, graph=False):
        import torch
        L = lib()
        s = (stream or torch.cuda.current_stream()).cuda_stream
        f = L.fg_plan_launch_graph if graph else L.fg_plan_launch
        f.argtypes = [_P, _P]
        st = f(self.handle, s)
        if st != FG_OK:
            raise FlashgemmError(st, last_error())

    def info(self):
        """dict(kernel, order, device_bytes, kernels, flops)."""
        L = lib()
        k, o, b, n, fl = ctypes.c_int(), ctypes.c_int(), _L(), ctypes.c_int(), ctypes.c_double()
        L.fg_plan_info.argtypes = [_P, _P, _P, _P, _P, _P]
        st = L.fg_plan_info(self.handle, ctypes.byref(k), ctypes.byref(o), ctypes.byref(b),
                            ctypes.byref(n), ctypes.byref(fl))
        if st != FG_OK:
            raise FlashgemmError(st, last_error())
        return dict(kernel=k.value, order=o.value, device_bytes=b.value, kernels=n.value,
                    flops=fl.value)

    def release(self):
        if self.handle:
            L = lib()
            L.fg_plan_release.argtypes = [_P]
            L.fg_plan_release(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.release()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass


# ---------------------------------------------------------------- serving loop

class _Request(ctypes.Structure):
    _fields_ = [("dtype", ctypes.c_int), ("num_gemm", ctypes.c_int), ("W", _P), ("N", _L),
                ("B", _P), ("C", _P), ("where", ctypes.c_int)]


class _ServerOpts(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_longlong), ("max_batch", ctypes.c_int),
                ("slots", ctypes.c_int), ("max_wait_us", ctypes.c_int),
                ("ctas_per_batch", ctypes.c_int), ("max_queue_us", ctypes.c_int)]


class _ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("completed", ctypes.c_longlong),
                ("failed", ctypes.c_longlong), ("shed", ctypes.c_longlong),
                ("batches", ctypes.c_longlong),
                ("mean_batch", ctypes.c_double), ("p50_us", ctypes.c_double),
                ("p99_us", ctypes.c_double), ("mean_us", ctypes.c_double),
                ("max_us", ctypes.c_double), ("flops", ctypes.c_double),
                ("span_s", ctypes.c_double), ("peak_bytes", ctypes.c_longlong)]


class Server:
    """The library's request loop (fg_server_*): chain requests on registered
    weights, admitted by device memory, batched into grouped launches."""

    def __init__(self, hbm_budget=0, max_batch=0, slots=0, max_wait_us=0, ctas_per_batch=0,
                 max_queue_us=0):
        L = lib()
        L.fg_server_create.argtypes = [_P, _P]
        L.fg_server_submit.argtypes = [_P, _P]
        L.fg_server_submit.restype = ctypes.c_longlong
        L.fg_server_wait.argtypes = [_P, ctypes.c_longlong, _P]
        L.fg_server_drain.argtypes = [_P]
        L.fg_server_get_stats.argtypes = [_P, _P]
        L.fg_server_reset_stats.argtypes = [_P]
        L.fg_server_destroy.argtypes = [_P]
        o = _ServerOpts(int(hbm_budget), int(max_batch), int(slots), int(max_wait_us),
                        int(ctas_per_batch), int(max_queue_us))
        h = _P()
        st = L.fg_server_create(ctypes.byref(o), ctypes.byref(h))
        if st != FG_OK:
            raise FlashgemmError(st, last_error())
        self.handle = h.value
        self._keep = {}

    def submit(self, dtype, weights, B, C, N=None):
        """Queue C = A_n ... A_1 B on `weights` (list of Weights). B and C are
        host numpy arrays or CUDA tensors (both the same kind); returns the id."""
        L = lib()
        host = isinstance(B, np.ndarray)
        N = int(B.shape[1] if N is None else N)
        hs = (_P * len(weights))(*[w.handle for w in weights])
        ptr = (lambda a: a.ctypes.data) if host else (lambda a: a.data_ptr())
        r = _Request(_DT[dtype], len(weights), ctypes.cast(hs, _P), N, ptr(B), ptr(C),
                     FG_MEM_HOST if host else FG_MEM_DEVICE)
        rid = L.fg_server_submit(self.handle, ctypes.byref(r))
        if rid < 0:
            raise FlashgemmError(-rid, last_error())
        self._keep[rid] = (hs, B, C, weights)
        return rid

    def wait(self, rid, shed_ok=False):
        """Blocks until request `rid` is done; returns its latency in microseconds.
        shed_ok: a request shed under load (FG_ERR_BUSY) returns None instead of
        raising."""
        L = lib()
        lat = ctypes.c_double()
        st = L.fg_server_wait(self.handle, ctypes.c_longlong(rid), ctypes.byref(lat))
        self._keep.pop(rid, None)
        if st == FG_ERR_BUSY and shed_ok:
            return None
        if st != FG_OK:
            raise FlashgemmError(st, last_error())
        return lat.value

    def replay(self, requests, at_us):
        """Submit requests [(dtype, weights, B, C), ...] at the given offsets
        (microseconds from now, non-decreasing) from native code; returns the ids."""
        L = lib()
        n = len(requests)
        arr = (_Request * n)()
        keep = []
        for r, (dtype, weights, B, C) in zip(arr, requests):
            host = isinstance(B, np.ndarray)
            hs = (_P * len(weights))(*[w.handle for w in weights])
            keep.append((hs, B, C, weights))
            r.dtype, r.num_gemm, r.W = _DT[dtype], len(weights), ctypes.cast(hs, _P)
            r.N = int(B.shape[1])
            r.B = B.ctypes.data if host else B.data_ptr()
            r.C = C.ctypes.data if host else C.data_ptr()
            r.where = FG_MEM_HOST if host else FG_MEM_DEVICE
        at = (ctypes.c_double * n)(*[float(x) for x in at_us])
        ids = (ctypes.c_longlong * n)()
        L.fg_server_replay.argtypes = [_P, _P, ctypes.c_int, _P, _P]
        st = L.fg_server_replay(self.handle, arr, n, at, ids)
        if st != FG_OK:
            raise FlashgemmError(st, last_error())
        out = list(ids)
        for rid, k in zip(out, keep):
            if rid >= 0:
                self._keep[rid] = k
        return out

    def drain(self):
        st = lib().fg_server_drain(self.handle)
        if st != FG_OK:
            raise FlashgemmError(st, last_error())

    def stats(self):
        s = _ServerStats()
        st = lib().fg_server_get_stats(self.handle, ctypes.byref(s))
        if st != FG_OK:
            raise FlashgemmError(st, last_error())
        return {k: getattr(s, k) for k, _ in _ServerStats._fields_}

    def reset_stats(self):
        lib().fg_server_reset_stats(self.handle)

    def close(self):
        if self.handle:
            lib().fg_server_destroy(self.handle)
            self.handle = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass
