"""The oracle pinned: the C restatement against the reference's own outputs.

Two sources of truth for the reference's behaviour:
  * the committed golden vectors in tests/golden/, produced by the reference
    compiled from its sources (tests/golden/make_golden.py), and
  * the reference itself (oracle/_ref), where it was built in this checkout.
"""
import glob
import os

import numpy as np
import pytest

import oracle

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _load(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def _chain_inputs(g):
    dt = str(g["dtype"])
    Ms = [int(x) for x in g["Ms"]]
    if "B" in g:
        B = g["B"]
        As = [g[f"A{i}"] for i in range(len(Ms))]
        Ks = [int(x) for x in g["Ks"]]
    else:
        B, As, Ks = oracle.chain_inputs(dt, int(g["N"]), int(g["K1"]), Ms, int(g["seed"]))
    return dt, B, As, Ms, Ks


@pytest.mark.parametrize("path", [p for p in GOLDEN if "_chain_" in p], ids=os.path.basename)
def test_chain_restatement_matches_golden(path):
    g = _load(path)
    dt, B, As, Ms, Ks = _chain_inputs(g)
    N = int(g["N"])
    C = np.zeros_like(g["C"])
    if dt == "int8":
        C[:] = int(g["sentinel"])
    oracle.chain(dt, B, As, N, Ms, Ks, mode=oracle.REF, threads=int(g["threads"]), C=C)
    # bit-exact for every dtype: the restatement follows the reference's own
    # accumulation order (vfmadd231ps / vdpbf16ps / vpdpbusd)
    np.testing.assert_array_equal(C, g["C"])


@pytest.mark.parametrize("path", [p for p in GOLDEN if "_sgemm_" in p], ids=os.path.basename)
def test_sgemm_restatement_matches_golden(path):
    g = _load(path)
    if "A" in g:
        A, B = g["A"], g["B"]
    else:
        A, B = oracle.sgemm_inputs(int(g["M"]), int(g["N"]), int(g["K"]), int(g["seed"]))
    np.testing.assert_array_equal(oracle.sgemm_f32(A, B, kblock=2048), g["C"])


def test_generators_reproduce_golden_inputs():
    """Fixtures stored without inputs rely on the seeded generators."""
    import hashlib
    for path in GOLDEN:
        g = _load(path)
        if "_sgemm_" in path:
            A, B = oracle.sgemm_inputs(int(g["M"]), int(g["N"]), int(g["K"]), int(g["seed"]))
            arrs = [A, B]
        else:
            dt = str(g["dtype"])
            B, As, _ = oracle.chain_inputs(dt, int(g["N"]), int(g["K1"]),
                                           [int(x) for x in g["Ms"]], int(g["seed"]))
            arrs = [B] + As
        h = hashlib.sha256()
        for a in arrs:
            h.update(np.ascontiguousarray(a).tobytes())
        assert h.hexdigest() == str(g["input_sha256"]), path


def test_math_mode_differs_from_ref_mode():
    """The reference's BF16/INT8 chains are not the mathematical chain."""
    B, As, Ks = oracle.chain_inputs("bf16", 64, 64, [32, 32], seed=3)
    r = oracle.chain("bf16", B, As, 64, [32, 32], Ks, mode=oracle.REF, threads=2)
    m = oracle.chain("bf16", B, As, 64, [32, 32], Ks, mode=oracle.MATH, threads=2)
    assert oracle.rel_frob(r, m) > 0.5
    # the MATH chain agrees with FP64 to BF16 precision
    Bf = oracle.bf16_to_f32(B)
    Af = [oracle.bf16_to_f32(a) for a in As]
    ref64 = oracle.chain_f64(Bf, Af, 64, [32, 32], Ks)
    assert oracle.rel_frob(m, ref64) < 1e-2


ref_only = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built here")


@ref_only
@pytest.mark.parametrize("dt", ["f32", "bf16", "int8"])
@pytest.mark.parametrize("shape", [
    (256, 64, [48, 96, 24], 8),
    (512, 128, [40, 20, 16], 8),
    (256, 64, [36, 28, 32], 8),
    (160, 64, [24, 24], 5),
    (256, 2048, [96, 48, 96, 24], 8),
])
def test_restatement_matches_live_reference(dt, shape):
    N, K1, Ms, T = shape
    B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=5)
    C1 = oracle.ref_chain(dt, B, As, N, Ms, Ks, threads=T)
    C2 = oracle.chain(dt, B, As, N, Ms, Ks, mode=oracle.REF, threads=T)
    mw = (Ms[-1] // 4) * 4 if dt == "int8" else Ms[-1]
    np.testing.assert_array_equal(C2[:mw], C1[:mw])


@ref_only
@pytest.mark.parametrize("shape", [(1024, 1024, 1024), (128, 2048, 4096), (512, 64, 128)])
def test_sgemm_restatement_matches_live_reference(shape):
    M, N, K = shape
    A, B = oracle.sgemm_inputs(M, N, K, seed=7)
    np.testing.assert_array_equal(oracle.sgemm_f32(A, B, kblock=2048), oracle.ref_sgemm(A, B))
