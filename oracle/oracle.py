"""Test infrastructure only: the oracle (never imported by the product path).

ctypes bindings for
  * liboracle.so            - the C restatement in fg_oracle.c, and
  * _ref/libref_*.so        - the reference compiled from its own sources by
                              oracle/Makefile (present where the reference was
                              built; absent means those helpers raise).
plus the seeded input generators shared by the tests, the golden-vector script
and bench.py's CPU-baseline leg, so that the reference, the restatement and the
B200 library always see the same bytes.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_P = ctypes.c_void_p
_L = ctypes.c_long

REF, MATH = 0, 1


def _ptr(a):
    return a.ctypes.data_as(_P)


def _parr(arrs):
    return (_P * len(arrs))(*[_ptr(a) for a in arrs])


def _larr(v):
    return (ctypes.c_long * len(v))(*[int(x) for x in v])


_lib = None


def lib():
    """Load liboracle.so (build it with `make -C oracle oracle`)."""
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle oracle`")
        _lib = ctypes.CDLL(path)
        _lib.orc_strip_width.restype = ctypes.c_long
        _lib.orc_strip_width.argtypes = [_L, ctypes.c_int]
    return _lib


_ref_m = None
_ref_s = None


def ref_available():
    return os.path.exists(os.path.join(REF_DIR, "libref_multigemm.so"))


def ref_multigemm():
    global _ref_m
    if _ref_m is None:
        _ref_m = ctypes.CDLL(os.path.join(REF_DIR, "libref_multigemm.so"))
    return _ref_m


def ref_singlegemm():
    global _ref_s
    if _ref_s is None:
        _ref_s = ctypes.CDLL(os.path.join(REF_DIR, "libref_singlegemm.so"))
        _ref_s.ref_set_thread_nums(24)  # FP32_ID23.c:68 (NUM = 24 is compiled into :35)
    return _ref_s


# ---------------------------------------------------------------- generators

def bf16_rne(x):
    """FP32 -> BF16 bits, round to nearest even."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = u + 0x7FFF + ((u >> 16) & 1)
    return (u >> 16).astype(np.uint16)


def bf16_to_f32(h):
    return (np.asarray(h, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def chain_inputs(dtype, N, K1, Ms, seed=0):
    """Seeded chain operands in the reference orientation.

    B: K1 x N, A_i: M_i x K_i with K_{i+1} = M_i.
      f32 : iid U[-1, 1]
      bf16: iid N(0,1) / sqrt(K_i), rounded to BF16 (B: N(0,1))
      int8: iid integers U[-127, 127] stored as bytes (B handed over as uint8,
            the reference's API type; its kernels read B signed, A unsigned)
    """
    rng = np.random.default_rng(seed)
    Ks = [K1] + list(Ms[:-1])
    if dtype == "f32":
        B = rng.uniform(-1, 1, (K1, N)).astype(np.float32)
        As = [rng.uniform(-1, 1, (m, k)).astype(np.float32) for m, k in zip(Ms, Ks)]
    elif dtype == "bf16":
        B = bf16_rne(rng.standard_normal((K1, N)))
        As = [bf16_rne(rng.standard_normal((m, k)) / np.sqrt(k)) for m, k in zip(Ms, Ks)]
    elif dtype == "int8":
        B = rng.integers(-127, 128, size=(K1, N)).astype(np.int8).view(np.uint8)
        As = [rng.integers(-127, 128, size=(m, k)).astype(np.int8) for m, k in zip(Ms, Ks)]
    else:
        raise ValueError(dtype)
    return B, As, Ks


def sgemm_inputs(M, N, K, seed=0):
    rng = np.random.default_rng(seed)
    A = rng.uniform(-1, 1, (M, K)).astype(np.float32)
    B = rng.uniform(-1, 1, (K, N)).astype(np.float32)
    return A, B


# ---------------------------------------------------------------- restatement

def chain(dtype, B, As, N, Ms, Ks, mode=REF, threads=8, C=None):
    """Run the C restatement of a chain; returns C (M_n x N)."""
    L = lib()
    n = len(As)
    if dtype == "f32":
        C = np.zeros((Ms[-1], N), np.float32) if C is None else C
        L.orc_chain_f32(_ptr(C), _ptr(B), _L(N), n, _parr(As), _larr(Ms), _larr(Ks))
    elif dtype == "bf16":
        C = np.zeros((Ms[-1], N), np.float32) if C is None else C
        rc = L.orc_chain_bf16(_ptr(C), _ptr(B), _L(N), n, _parr(As), _larr(Ms), _larr(Ks),
                              mode, threads)
        assert rc == 0
    elif dtype == "int8":
        C = np.zeros((Ms[-1], N), np.int32) if C is None else C
        rc = L.orc_chain_int8(_ptr(C), _ptr(B), _L(N), n, _parr(As), _larr(Ms), _larr(Ks),
                              mode, threads)
        assert rc == 0
    else:
        raise ValueError(dtype)
    return C


def chain_f64(B, As, N, Ms, Ks):
    C = np.zeros((Ms[-1], N), np.float64)
    lib().orc_chain_f64(_ptr(C), _ptr(B), _L(N), len(As), _parr(As), _larr(Ms), _larr(Ks))
    return C


def sgemm_f32(A, B, kblock=2048):
    M, K = A.shape
    N = B.shape[1]
    C = np.zeros((M, N), np.float32)
    lib().orc_sgemm_f32(_ptr(A), _ptr(B), _ptr(C), _L(M), _L(N), _L(K), _L(kblock))
    return C


def sgemm_f64(A, B):
    M, K = A.shape
    N = B.shape[1]
    C = np.zeros((M, N), np.float64)
    lib().orc_sgemm_f64(_ptr(A), _ptr(B), _ptr(C), _L(M), _L(N), _L(K))
    return C


def strip_width(N, threads):
    return int(lib().orc_strip_width(N, threads))


def rel_frob(x, ref):
    x = np.asarray(x, np.float64)
    ref = np.asarray(ref, np.float64)
    den = np.linalg.norm(ref)
    return float(np.linalg.norm(x - ref) / (den if den > 0 else 1.0))


# ---------------------------------------------------------------- the reference

def ref_chain(dtype, B, As, N, Ms, Ks, threads=8, C=None):
    """Run the reference's own flashgemm_multi_* (compiled from its sources)."""
    R = ref_multigemm()
    R.ref_set_threads(int(threads))
    n = len(As)
    fn = {"f32": R.ref_chain_f32, "bf16": R.ref_chain_bf16, "int8": R.ref_chain_int8}[dtype]
    if C is None:
        C = np.zeros((Ms[-1], N), np.int32 if dtype == "int8" else np.float32)
    rc = fn(_ptr(C), _ptr(B), _L(N), n, _parr(As), _larr(Ms), _larr(Ks))
    assert rc == 0
    return C


def ref_sgemm(A, B, threads=None):
    """The reference's singlegemm. threads=None: LibShalom_sgemm_mp as compiled
    (NUM = 24); else Small_NGM_NN_SGEMM / Small_MGN_NN_SGEMM with that many
    threads on the grid Dete_grad_N_threads_nums picks (FP32_ID23.c:47-60)."""
    S = ref_singlegemm()
    M, K = A.shape
    N = B.shape[1]
    C = np.zeros((M, N), np.float32)
    if threads is None:
        S.ref_reset_thread_nums(24)
        S.ref_sgemm_mp(0, 0, _ptr(C), _ptr(A), _ptr(B), _L(M), _L(N), _L(K))
        return C
    S.ref_reset_thread_nums(int(threads))
    if M // N >= 8:
        S.ref_sgemm_mgn(_ptr(C), _ptr(A), _ptr(B), _L(M), _L(N), _L(K), threads, threads, 1)
    else:
        tm, tn = ctypes.c_int(), ctypes.c_int()
        S.ref_dete_grad_n(threads, _L(M), _L(N), ctypes.byref(tm), ctypes.byref(tn))
        S.ref_sgemm_ngm(_ptr(C), _ptr(A), _ptr(B), _L(M), _L(N), _L(K), threads, tm.value,
                        tn.value)
    return C
