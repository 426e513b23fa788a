"""Grouped launches: many chains of uneven lengths and shapes in one launch.

Every kernel / stage-order candidate of the grouped path is checked against
the same chains run one by one through the single-chain entry point, and
against the oracle (the reference's semantics): INT8 bit-exact, BF16 within the
BF16 tolerance of the reference, FP32 3xTF32 within 2x the plain FP32 kernel's
own error against FP64 (and plain FP32 bit-exact with the reference's FMA
order). Plans are checked to replay identically through a CUDA graph, and the
autotuner to return and remember a valid choice.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

BF16_TOL = 2e-3  # the BF16 tolerance of the parity tests (against the reference semantics)
PAIR, S256, S128 = 0, 1, 2
FUSED, LEVELS = 0, 1


@pytest.fixture(scope="module", autouse=True)
def fg():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import flashgemm_b200 as fg
    fg.lib()
    fg.set_semantics("ref")
    fg.set_f32_algo("3xtf32")
    yield fg
    fg.set_group_config(-1, -1)
    fg.set_semantics("ref")
    fg.set_f32_algo("3xtf32")


def _specs(dt, seed, count, dims=(64, 128, 272, 520, 1024), widths=(128, 260, 384, 1000),
           Ns=(256, 512, 768, 1280), lengths=(2, 5)):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(lengths[0], lengths[1]))
        N = int(rng.choice(Ns))
        K1 = int(rng.choice(dims))
        Ms = [int(rng.choice(widths)) for _ in range(n)]
        if dt == "int8":
            K1 = max(64, K1 // 32 * 32)
        out.append((N, K1, Ms))
    return out


def _torch(a):
    import torch
    if a.dtype == np.uint8:
        a = a.view(np.int8)
    elif a.dtype == np.uint16:
        a = a.view(np.int16)
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _build(fg, dt, specs, seed0):
    """Registered weights, device inputs, and (alone, grouped) output buffers."""
    import torch
    chains, alone, host = [], [], []
    for j, (N, K1, Ms) in enumerate(specs):
        B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=seed0 + j)
        W = [fg.Weights(dt, a) for a in As]
        tB = _torch(B)
        odt = torch.int32 if dt == "int8" else torch.float32
        c1 = torch.zeros((Ms[-1], N), dtype=odt, device="cuda")
        c2 = torch.full((Ms[-1], N), 7, dtype=odt, device="cuda")
        fg.chain_registered(dt, c1, tB, N, W)
        chains.append((c2, tB, N, W))
        alone.append(c1)
        host.append((B, As, Ks))
    return chains, alone, host


def _release(chains):
    for _, _, _, W in chains:
        for w in W:
            w.release()


def _rows_written(dt, M):
    # INT8 reference semantics leave the last M % 4 rows of C untouched
    return (M // 4) * 4 if dt == "int8" else M


@pytest.mark.parametrize("order", [FUSED, LEVELS])
@pytest.mark.parametrize("kernel", [PAIR, S256, S128])
@pytest.mark.parametrize("dt", ["int8", "bf16"])
def test_group_candidates_match_chains_alone(fg, dt, kernel, order):
    import torch
    fg.set_group_config(kernel, order)
    try:
        chains, alone, _ = _build(fg, dt, _specs(dt, 11 + kernel, 9), 300)
        assert fg.group_choice(dt, chains) == (kernel, order)
        fg.chain_group(dt, chains)
        torch.cuda.synchronize()
        fg.sync()
        for (c2, _, _, _), c1 in zip(chains, alone):
            r = _rows_written(dt, c1.shape[0])
            np.testing.assert_array_equal(c2[:r].cpu().numpy(), c1[:r].cpu().numpy())
        _release(chains)
    finally:
        fg.set_group_config(-1, -1)


@pytest.mark.parametrize("kernel", [S256, S128])
@pytest.mark.parametrize("dt", ["int8", "bf16"])
def test_single_cta_group_matches_reference(fg, dt, kernel):
    """Single-CTA kernels against the oracle (the reference's semantics,
    including the INT8 tail rows and the BF16 / INT8 panel permutation)."""
    import torch
    fg.set_group_config(kernel, FUSED)
    try:
        specs = [(256, 256, [300, 136]), (512, 128, [1000, 520, 264]), (128, 520, [76, 128])]
        chains, _, host = _build(fg, dt, specs, 500)
        fg.chain_group(dt, chains)
        torch.cuda.synchronize()
        fg.sync()
        for (c2, _, N, _), (B, As, Ks), (_, _, Ms) in zip(chains, host, specs):
            want = oracle.chain(dt, B, As, N, Ms, Ks, mode=oracle.REF, threads=1)
            got = c2.cpu().numpy()
            r = _rows_written(dt, Ms[-1])
            if dt == "int8":
                np.testing.assert_array_equal(got[:r], want[:r])
            else:
                assert oracle.rel_frob(got, want) <= BF16_TOL
        _release(chains)
    finally:
        fg.set_group_config(-1, -1)


@pytest.mark.parametrize("order", [FUSED, LEVELS])
def test_group_f32_3xtf32_matches_alone_and_fp64(fg, order):
    import torch
    fg.set_group_config(S128, order)
    fg.set_f32_algo("3xtf32")
    try:
        specs = _specs("f32", 21, 8, dims=(64, 128, 272, 1024), widths=(64, 128, 260, 512),
                       Ns=(64, 128, 320, 512))
        chains, alone, host = _build(fg, "f32", specs, 700)
        fg.chain_group("f32", chains)
        torch.cuda.synchronize()
        fg.sync()
        fg.set_f32_algo("ffma")
        plain = []
        for (c2, tB, N, W) in chains:
            c3 = torch.zeros_like(c2)
            fg.chain_registered("f32", c3, tB, N, W)
            plain.append(c3)
        torch.cuda.synchronize()
        for (c2, _, N, _), c1, c3, (B, As, Ks) in zip(chains, alone, plain, host):
            got = c2.cpu().numpy()
            np.testing.assert_array_equal(got, c1.cpu().numpy())
            exact = oracle.chain_f64(B, As, N, [a.shape[0] for a in As], Ks)
            e3 = oracle.rel_frob(got, exact)
            ef = oracle.rel_frob(c3.cpu().numpy(), exact)
            assert e3 <= 2.0 * ef + 1e-12, (e3, ef)
        _release(chains)
    finally:
        fg.set_f32_algo("3xtf32")
        fg.set_group_config(-1, -1)


def test_group_f32_ffma_bit_exact(fg):
    """Plain FP32 groups (one grouped CUDA-core launch per chain depth) give
    exactly the single-chain FMA results, which are bit-exact with the
    reference's FP32 chain (multigemm/src/kernel_f32.h)."""
    import torch
    fg.set_f32_algo("ffma")
    try:
        specs = _specs("f32", 31, 10, dims=(64, 128, 272, 1024), widths=(64, 128, 260, 512),
                       Ns=(64, 128, 320, 512))
        chains, alone, host = _build(fg, "f32", specs, 800)
        fg.chain_group("f32", chains)
        torch.cuda.synchronize()
        fg.sync()
        for (c2, _, N, _), c1, (B, As, Ks), (_, _, Ms) in zip(chains, alone, host, specs):
            got = c2.cpu().numpy()
            np.testing.assert_array_equal(got, c1.cpu().numpy())
        # one chain against the oracle's FMA restatement of the reference
        (c2, _, N, _), (B, As, Ks), (_, _, Ms) = chains[0], host[0], specs[0]
        np.testing.assert_array_equal(c2.cpu().numpy(), oracle.chain("f32", B, As, N, Ms, Ks))
        _release(chains)
    finally:
        fg.set_f32_algo("3xtf32")


@pytest.mark.parametrize("dt", ["bf16", "int8", "f32"])
def test_plan_graph_replays_group(fg, dt):
    """A plan launched directly and replayed through its CUDA graph gives the
    grouped launch's results; graph replays run the same kernels."""
    import torch
    specs = _specs(dt, 41, 6, Ns=(256, 512))
    chains, alone, _ = _build(fg, dt, specs, 900)
    fg.chain_group(dt, chains)
    torch.cuda.synchronize()
    want = [c[0].clone() for c in chains]
    for c in chains:
        c[0].fill_(3)
    plan = fg.Plan(dt, chains)
    info = plan.info()
    assert info["kernels"] >= 1 and info["device_bytes"] > 0 and info["flops"] > 0
    plan.launch()
    torch.cuda.synchronize()
    for c, w in zip(chains, want):
        assert torch.equal(c[0], w)
        c[0].fill_(5)
    for _ in range(3):
        plan.launch(graph=True)
    torch.cuda.synchronize()
    fg.sync()
    for c, w in zip(chains, want):
        assert torch.equal(c[0], w)
    plan.release()
    _release(chains)


def test_autotuner_measures_and_remembers(fg, tmp_path):
    import torch
    specs = _specs("bf16", 51, 5, Ns=(256, 512))
    chains, alone, _ = _build(fg, "bf16", specs, 1000)
    k, o, ms = fg.autotune_group("bf16", chains, iters=2)
    assert k in (PAIR, S256, S128) and o in (FUSED, LEVELS) and ms > 0
    assert fg.group_choice("bf16", chains) == (k, o)
    path = tmp_path / "tune.txt"
    fg.autotune_save(path)
    assert path.read_text().strip()
    fg.chain_group("bf16", chains)
    torch.cuda.synchronize()
    fg.sync()
    for (c2, _, _, _), c1 in zip(chains, alone):
        assert torch.equal(c2, c1)
    _release(chains)


def test_large_group_many_stages(fg):
    """Hundreds of chains (stage tables far beyond the kernel parameters) with
    small dimensions from 64: every chain equals its single-chain result."""
    import torch
    rng = np.random.default_rng(61)
    specs = []
    for _ in range(160):
        n = int(rng.integers(2, 6))
        dims = [int(16 * round(np.exp(rng.uniform(np.log(64), np.log(1024))) / 16)) for _ in range(n + 1)]
        specs.append((int(rng.choice([64, 128, 256])), dims[0], dims[1:]))
    for dt in ("bf16", "int8"):
        chains, alone, _ = _build(fg, dt, specs, 1100)
        fg.chain_group(dt, chains)
        torch.cuda.synchronize()
        fg.sync()
        for (c2, _, _, _), c1 in zip(chains, alone):
            r = _rows_written(dt, c1.shape[0])
            assert torch.equal(c2[:r], c1[:r])
        _release(chains)
