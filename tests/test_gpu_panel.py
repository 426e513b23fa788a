"""FP32 chains whose every dimension fits on chip run panel-resident: one launch,
B read once, each stage's (hi, lo) TF32 operand handed to the next stage in
shared memory (the reference's flashgemm.c:123-148 keeps its panel in a
per-thread buffer the same way). The arithmetic is the 3xTF32 stage kernels',
so these tests check bit equality with the per-stage path (one launch per GEMM,
intermediates through global memory) and the accuracy contract against FP64:
within 2x the plain FP32 kernel's own error.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

PANEL_SHAPES = [
    # N, K1, Ms   (every dimension <= 64)
    (65536, 64, [64, 64, 64]),      # the tall-skinny grouped workload's shape
    (4100, 48, [40, 64, 18]),       # ragged: N % 128 != 0, K and M not multiples of 32
    (256, 64, [64]),                # one stage
    (1024, 16, [8, 64, 32, 64, 24]),  # five stages, K < 32
]


@pytest.fixture(scope="module", autouse=True)
def fg():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import flashgemm_b200 as fg
    fg.lib()
    fg.set_semantics("ref")
    fg.set_f32_algo("3xtf32")
    fg.set_chain_mode("fused")
    yield fg
    fg.set_f32_algo("3xtf32")
    fg.set_chain_mode("fused")


def _run(fg, B, As, N, Ms, Ks):
    C = np.zeros((Ms[-1], N), np.float32)
    trip = []
    for A, m, k in zip(As, Ms, Ks):
        trip += [A, m, k]
    fg.flashgemm_multi_f32f32f32(C, B, N, len(As), *trip, check=True)
    return C


@pytest.mark.parametrize("shape", PANEL_SHAPES, ids=lambda s: f"n{s[0]}_k{s[1]}_" + "-".join(map(str, s[2])))
def test_panel_chain_equals_per_stage_path_and_meets_accuracy(fg, shape):
    N, K1, Ms = shape
    rng = np.random.default_rng(N + K1)
    Ks = [K1] + Ms[:-1]
    B = rng.standard_normal((K1, N)).astype(np.float32)
    As = [(rng.standard_normal((m, k)) / np.sqrt(k)).astype(np.float32) for m, k in zip(Ms, Ks)]
    launches = fg.kernel_launches()
    panel = _run(fg, B, As, N, Ms, Ks)
    # weights split + one panel launch, whatever the chain's length
    assert fg.kernel_launches() - launches <= len(Ms) + 1
    fg.set_chain_mode("per_gemm")
    try:
        stages = _run(fg, B, As, N, Ms, Ks)
    finally:
        fg.set_chain_mode("fused")
    np.testing.assert_array_equal(panel, stages)
    exact = oracle.chain_f64(B, As, N, Ms, Ks)
    plain = oracle.chain("f32", B, As, N, Ms, Ks)
    e_panel, e_plain = oracle.rel_frob(panel, exact), oracle.rel_frob(plain, exact)
    assert e_panel <= 2 * e_plain, (e_panel, e_plain)


def test_group_with_panel_chains_matches_chains_run_alone(fg):
    """Tall-skinny chains (panel-resident) and wider ones (the grouped kernel)
    in one grouped launch give exactly what each gives alone."""
    import torch
    specs = [(65536, 64, [64, 64]), (8192, 256, [512, 128]), (4096, 64, [64, 64, 64, 64]),
             (1024, 96, [64, 200]), (2048, 32, [48, 64, 16])]
    chains, alone, keep = [], [], []
    for j, (N, K1, Ms) in enumerate(specs):
        rng = np.random.default_rng(300 + j)
        Ks = [K1] + Ms[:-1]
        B = rng.standard_normal((K1, N)).astype(np.float32)
        As = [(rng.standard_normal((m, k)) / np.sqrt(k)).astype(np.float32) for m, k in zip(Ms, Ks)]
        W = [fg.Weights("f32", a) for a in As]
        tB = torch.from_numpy(B).cuda()
        c1 = torch.zeros((Ms[-1], N), device="cuda")
        c2 = torch.zeros((Ms[-1], N), device="cuda")
        fg.set_chain_mode("per_gemm")
        try:
            fg.chain_registered("f32", c1, tB, N, W)
        finally:
            fg.set_chain_mode("fused")
        chains.append((c2, tB, N, W))
        alone.append(c1)
        keep.append((B, As, N, Ms, Ks))
    fg.chain_group("f32", chains)
    torch.cuda.synchronize()
    fg.sync()
    for (c2, _, _, W), c1, (B, As, N, Ms, Ks) in zip(chains, alone, keep):
        np.testing.assert_array_equal(c2.cpu().numpy(), c1.cpu().numpy())
        for w in W:
            w.release()
