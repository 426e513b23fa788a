"""Parity on the reference's own shape tables, at full size, through the C ABI.

The reference's test programs time fixed tables of shapes:
  * multigemm/test/test_{f32,bf16,int8}.c:14-24  - 20 single GEMMs (M, N, K),
  * multigemm/test/test_{f32,bf16,int8}_3.c:14-48 - 10 three-stage chains
    (M1, N, K1), (M2, N, K2 = M1), (M3, N, K3 = M2),
  * singlegemm/FP32_ID23.c:11-33                - 23 SGEMM shapes (M, N, K).
They check nothing themselves (the checks are commented out), so here every
shape runs through this library's reference-named entry points at its full
size and is checked on a sample of its output against the oracle:
  * chains and single GEMMs: whole 32-column panels (the reference's panel
    permutation never crosses a panel, so panel p of C depends only on panel p
    of B) - bit-exact for INT8 and the plain FP32 kernel, relative Frobenius
    error <= BF16_TOL for BF16, and 3xTF32 FP32 within 2x the plain kernel's
    error against FP64;
  * SGEMM: a sample of whole rows, bit-exact (one FMA per k in increasing k,
    K cut into blocks of 2048 as singlegemm/src/NN_mp.h:13 does).
Where the compiled reference is present (oracle/_ref) and defined on the input
(INT8 needs K1 % 32 == 0; multigemm/src/flashgemm.c:71-75 packs B in 32-row
groups), the same panels are also checked against the reference itself.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

BF16_TOL = 2e-3

# multigemm/test/test_int8.c:13-23 (the same table in test_f32.c and test_bf16.c): M, N, K
SINGLE = [
    (32, 65536, 288), (24, 65536, 32), (144, 16384, 1296), (32, 16384, 144),
    (192, 16384, 1728), (32, 16384, 192), (192, 4096, 4800), (56, 4096, 192),
    (336, 4096, 8400), (56, 4096, 336), (32, 50176, 288), (16, 50176, 32),
    (96, 12544, 864), (24, 12544, 96), (144, 12544, 1296), (24, 12544, 144),
    (144, 3136, 1296), (32, 3136, 144), (192, 3136, 1728), (32, 3136, 192),
]

# multigemm/test/test_f32_3.c:14-48 (and test_bf16_3.c, test_int8_3.c): N, K1, (M1, M2, M3)
CHAINS = [
    (65536, 288, (32, 24, 144)), (16384, 1296, (144, 32, 192)), (16384, 1728, (192, 32, 192)),
    (4096, 4800, (192, 56, 336)), (4096, 8400, (336, 56, 336)), (50176, 288, (32, 16, 96)),
    (12544, 864, (96, 24, 144)), (12544, 1296, (144, 24, 144)), (3136, 1296, (144, 32, 192)),
    (3136, 1728, (192, 32, 192)),
]

# singlegemm/FP32_ID23.c:11-33: M, N, K
SGEMM = [
    (128, 2048, 4096), (320, 3072, 4096), (1632, 36548, 1024), (2048, 4096, 32),
    (31999, 1024, 80), (84, 1024, 4096), (256, 256, 2048), (1024, 16, 500000),
    (35, 8457, 2560), (64, 18496, 128), (128, 4624, 256), (256, 1156, 512),
    (512, 289, 1024), (256, 3136, 64), (64, 3136, 64), (64, 3136, 256),
    (512, 784, 128), (128, 784, 512), (32, 16384, 288), (144, 4096, 1296),
    (144, 1024, 1296), (192, 1024, 1728), (96, 4096, 864),
]


@pytest.fixture(scope="module", autouse=True)
def fg():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import flashgemm_b200 as fg
    fg.lib()
    fg.set_semantics("ref")
    fg.set_f32_algo("3xtf32")
    fg.set_sgemm_algo("ffma")
    fg.flashgemm_set_thread_num(1)
    yield fg
    fg.set_f32_algo("3xtf32")


def _run(fg, dt, B, As, N, Ms, Ks):
    C = np.zeros((Ms[-1], N), np.int32 if dt == "int8" else np.float32)
    trip = []
    for A, m, k in zip(As, Ms, Ks):
        trip += [A, m, k]
    fn = {"f32": fg.flashgemm_multi_f32f32f32, "bf16": fg.flashgemm_multi_bf16bf16f32,
          "int8": fg.flashgemm_multi_int8uint8int32}[dt]
    fn(C, B, N, len(As), *trip, check=True)
    return C


def _panels(N):
    """Four whole 32-column panels: both ends and two inside."""
    last = N // 32 - 1
    ps = sorted({0, 1, last // 2, last})
    return np.concatenate([np.arange(32 * p, 32 * p + 32) for p in ps])


def _ref_usable():
    if not oracle.ref_available():
        return False
    flags = set()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    break
    except OSError:
        return False
    return {"avx512f", "avx512bw", "avx512_vnni", "avx512_bf16"} <= flags


def _check_chain(fg, dt, N, K1, Ms, seed):
    Ms = list(Ms)
    B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=seed)
    cols = _panels(N)
    Bs = np.ascontiguousarray(B[:, cols])
    if dt == "f32":
        fg.set_f32_algo("ffma")
        try:
            plain = _run(fg, dt, B, As, N, Ms, Ks)[:, cols]
        finally:
            fg.set_f32_algo("3xtf32")
        tf = _run(fg, dt, B, As, N, Ms, Ks)[:, cols]
        np.testing.assert_array_equal(plain, oracle.chain("f32", Bs, As, len(cols), Ms, Ks))
        exact = oracle.chain_f64(Bs, As, len(cols), Ms, Ks)
        e_plain, e_tf = oracle.rel_frob(plain, exact), oracle.rel_frob(tf, exact)
        assert e_tf <= 2 * e_plain, (e_tf, e_plain)
        got = plain
    else:
        got = np.ascontiguousarray(_run(fg, dt, B, As, N, Ms, Ks)[:, cols])
        want = oracle.chain(dt, Bs, As, len(cols), Ms, Ks, mode=oracle.REF, threads=1)
        if dt == "int8":
            np.testing.assert_array_equal(got, want)
        else:
            assert oracle.rel_frob(got, want) <= BF16_TOL
    # the reference itself on the same panels (one thread: panels start at multiples of 32)
    if _ref_usable() and not (dt == "int8" and K1 % 32):
        ref = oracle.ref_chain(dt, Bs, As, len(cols), Ms, Ks, threads=1)
        if dt == "bf16":
            assert oracle.rel_frob(got, ref) <= BF16_TOL
        else:
            np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("dt", ["int8", "bf16", "f32"])
@pytest.mark.parametrize("shape", SINGLE, ids=[f"{m}x{n}x{k}" for m, n, k in SINGLE])
def test_reference_single_gemm_table(fg, dt, shape):
    M, N, K = shape
    _check_chain(fg, dt, N, K, [M], seed=M * 7 + K)


@pytest.mark.parametrize("dt", ["int8", "bf16", "f32"])
@pytest.mark.parametrize("shape", CHAINS, ids=[f"n{n}_k{k}_" + "-".join(map(str, ms))
                                               for n, k, ms in CHAINS])
def test_reference_three_stage_chain_table(fg, dt, shape):
    N, K1, Ms = shape
    _check_chain(fg, dt, N, K1, Ms, seed=N + K1)


def _sgemm_inputs(M, N, K, seed):
    # float32 draws directly (the K = 500000 shape's A alone is 2 GB)
    rng = np.random.default_rng(seed)
    A = rng.random((M, K), dtype=np.float32) * 2 - 1
    B = rng.random((K, N), dtype=np.float32) * 2 - 1
    return A, B


@pytest.mark.parametrize("shape", SGEMM, ids=[f"{m}x{n}x{k}" for m, n, k in SGEMM])
def test_reference_sgemm_table_bitexact(fg, shape):
    M, N, K = shape
    A, B = _sgemm_inputs(M, N, K, seed=M + N + K)
    C = np.zeros((M, N), np.float32)
    fg.LibShalom_sgemm_mp(0, 0, C, A, B, M, N, K, check=True)
    rows = sorted({0, 1, M // 2, M - 2, M - 1} - {-1})
    want = oracle.sgemm_f32(np.ascontiguousarray(A[rows]), B, kblock=2048)
    np.testing.assert_array_equal(C[rows], want)
    assert np.isfinite(C).all()
