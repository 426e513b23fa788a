"""BF16 / INT8 chains whose intermediates have at most 256 rows run with the
intermediates on chip: each stage's result narrowed as the reference narrows it
(BF16 round-to-nearest-even or int8 saturation, the 2 x 32 / 4 x 32 panel
permutation, the INT8 tail rows) and written into shared memory as the next
stage's operand, as multigemm/src/flashgemm.c:123-148 keeps its panel in a
per-thread buffer. The products and their order are the other kernels', so the
result must equal the per-GEMM path (one launch per stage, intermediates through
global memory) bit for bit, and the oracle: INT8 exactly, BF16 within the
parity tolerance."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

BF16_TOL = 2e-3

SHAPES = [
    # N, K1, Ms
    (4096, 1024, [200, 56, 336]),        # two row tiles in stage 0; last stage three
    (1000, 520, [40, 24, 100, 36]),      # ragged N; INT8 tail rows in every stage
    (520, 64, [256, 256, 8]),            # full 256-row intermediates
    (3136, 1728, [192, 32, 192]),        # a shape of the reference's own chain table
    (65536, 288, [32, 24, 144]),         # the reference table's widest chain
]


@pytest.fixture(scope="module", autouse=True)
def fg():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import flashgemm_b200 as fg
    fg.lib()
    fg.set_semantics("ref")
    fg.set_chain_mode("fused")
    fg.set_narrow("always")  # the narrow kernel even where the fused one is faster
    fg.flashgemm_set_thread_num(1)
    yield fg
    fg.set_semantics("ref")
    fg.set_chain_mode("fused")
    fg.set_narrow("auto")


def _run(fg, dt, B, As, N, Ms, Ks):
    C = np.zeros((Ms[-1], N), np.int32 if dt == "int8" else np.float32)
    trip = []
    for A, m, k in zip(As, Ms, Ks):
        trip += [A, m, k]
    fn = {"bf16": fg.flashgemm_multi_bf16bf16f32, "int8": fg.flashgemm_multi_int8uint8int32}[dt]
    fn(C, B, N, len(As), *trip, check=True)
    return C


def _panels(N):
    last = N // 32 - 1
    ps = sorted({0, 1, last // 2, last})
    return np.concatenate([np.arange(32 * p, 32 * p + 32) for p in ps])


@pytest.mark.parametrize("sem", ["ref", "math"])
@pytest.mark.parametrize("dt", ["int8", "bf16"])
@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: f"n{s[0]}_k{s[1]}_" + "-".join(map(str, s[2])))
def test_narrow_chain_equals_per_gemm_and_oracle(fg, dt, sem, shape):
    N, K1, Ms = shape
    B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=N + K1 + len(Ms))
    fg.set_semantics(sem)
    try:
        launches = fg.kernel_launches()
        narrow = _run(fg, dt, B, As, N, Ms, Ks)
        used = fg.kernel_launches() - launches
        fg.set_chain_mode("per_gemm")
        try:
            per_gemm = _run(fg, dt, B, As, N, Ms, Ks)
        finally:
            fg.set_chain_mode("fused")
    finally:
        fg.set_semantics("ref")
    # one chain kernel per column chunk of the host call (plus INT8 tail preparation)
    assert used <= 8
    np.testing.assert_array_equal(narrow, per_gemm)
    rows = (Ms[-1] // 4) * 4 if dt == "int8" and sem == "ref" else Ms[-1]
    cols = _panels(N) if N > 4096 else np.arange(N)
    if N % 32 and N > 4096:
        cols = cols[cols < N]
    Bs = np.ascontiguousarray(B[:, cols])
    mode = oracle.REF if sem == "ref" else oracle.MATH
    want = oracle.chain(dt, Bs, As, len(cols), Ms, Ks, mode=mode, threads=1)
    got = np.ascontiguousarray(narrow[:, cols])
    if dt == "int8":
        np.testing.assert_array_equal(got[:rows], want[:rows])
    else:
        assert oracle.rel_frob(got, want) <= BF16_TOL
