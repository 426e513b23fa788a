"""Parity of the B200 path with the reference, through the C ABI.

Every computation here goes through libflashgemm_b200.so's reference-named
entry points (flashgemm_multi_*, LibShalom_sgemm_mp) or its device entry
points, and is checked against the oracle: the committed golden vectors the
reference produced, the C restatement of the reference (bit-exact with it), and
an FP64 evaluation for accuracy statements.

Tolerances (stated per dtype, as in the contract for this path):
  INT8  bit-exact against the reference semantics;
  BF16  relative Frobenius error <= 2e-3 against the reference semantics
        (at most 6.3e-4 measured over every chain and reference shape of these
        tests: FP32 accumulation order differs from vdpbf16ps, which flips a
        few BF16 roundings between stages);
  FP32  plain-FMA kernel bit-exact; 3xTF32 within 2x the plain kernel's own
        error against FP64.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

BF16_TOL = 2e-3
# BF16 chain against the exact (FP64, unrounded) chain: an accuracy statement, not
# parity; each between-stage narrowing to BF16 contributes up to 2^-9 relative
BF16_VS_FP64 = 1e-2


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
    fg.set_semantics("ref")
    fg.set_f32_algo("3xtf32")
    fg.set_sgemm_algo("ffma")
    fg.flashgemm_set_thread_num(1)


def run_chain(fg, dt, B, As, N, Ms, Ks, C=None, threads=1):
    fg.flashgemm_set_thread_num(threads)
    if C is None:
        C = np.zeros((Ms[-1], N), np.int32 if dt == "int8" else np.float32)
    trip = []
    for A, m, k in zip(As, Ms, Ks):
        trip += [A, m, k]
    fn = {"f32": fg.flashgemm_multi_f32f32f32, "bf16": fg.flashgemm_multi_bf16bf16f32,
          "int8": fg.flashgemm_multi_int8uint8int32}[dt]
    fn(C, B, N, len(As), *trip, check=True)
    return C


def assert_parity(dt, got, want, rows=None):
    if rows is not None:
        got, want = got[:rows], want[:rows]
    if dt == "int8":
        np.testing.assert_array_equal(got, want)
    else:
        err = oracle.rel_frob(got, want)
        assert err <= BF16_TOL if dt == "bf16" else err <= 1e-5, err


# ---------------------------------------------------------------- single stages (MATH)

@pytest.mark.parametrize("dt", ["int8", "bf16", "f32"])
@pytest.mark.parametrize("shape", [(128, 256, 128), (200, 96, 64), (64, 512, 256), (300, 520, 96)])
def test_single_stage_matches_oracle(fg, dt, shape):
    M, N, K = shape
    B, As, Ks = oracle.chain_inputs(dt, N, K, [M], seed=M + N)
    fg.set_semantics("math")
    try:
        got = run_chain(fg, dt, B, As, N, [M], Ks)
    finally:
        fg.set_semantics("ref")
    if dt == "f32":
        want = oracle.chain_f64(B, As, N, [M], Ks)
        assert oracle.rel_frob(got, want) < 2e-6
    else:
        want = oracle.chain(dt, B, As, N, [M], Ks, mode=oracle.MATH)
        assert_parity(dt, got, want)


# ---------------------------------------------------------------- golden vectors

def _golden(name):
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    return {k: z[k] for k in z.files}


@pytest.mark.parametrize("name", ["int8_chain_3stage", "int8_chain_tails", "int8_chain_c3_widths",
                                  "int8_chain_unwritten_rows", "bf16_chain_3stage",
                                  "bf16_chain_tails", "f32_chain_n96"])
def test_chain_matches_reference_golden(fg, name):
    g = _golden(name)
    dt = str(g["dtype"])
    Ms = [int(x) for x in g["Ms"]]
    Ks = [int(x) for x in g["Ks"]]
    B = g["B"]
    As = [g[f"A{i}"] for i in range(len(Ms))]
    N = int(g["N"])
    C = np.zeros_like(g["C"])
    if dt == "int8":
        C[:] = int(g["sentinel"])  # rows the reference never writes must stay untouched
    got = run_chain(fg, dt, B, As, N, Ms, Ks, C=C, threads=int(g["threads"]))
    if dt == "f32":
        want64 = oracle.chain_f64(B, As, N, Ms, Ks)
        e_ref = oracle.rel_frob(g["C"], want64)
        assert oracle.rel_frob(got, want64) <= 2 * e_ref + 1e-7
    else:
        assert_parity(dt, got, g["C"])


@pytest.mark.parametrize("name", ["f32_sgemm_96x128x64", "f32_sgemm_ksplit_48x128x2080",
                                  "f32_sgemm_mgn_768x64x96"])
def test_sgemm_matches_reference_golden_bitexact(fg, name):
    g = _golden(name)
    M, N, K = int(g["M"]), int(g["N"]), int(g["K"])
    if "A" in g:
        A, B = g["A"], g["B"]
    else:
        A, B = oracle.sgemm_inputs(M, N, K, int(g["seed"]))
    C = np.zeros((M, N), np.float32)
    fg.LibShalom_sgemm_mp(0, 0, C, A, B, M, N, K, check=True)
    np.testing.assert_array_equal(C, g["C"])


# ---------------------------------------------------------------- seeded sweeps

CHAIN_SHAPES = [
    # N, K1, Ms        (M % 12 in {0, 4, 8}, several M and N tiles, K not a multiple of 128)
    (256, 64, [48, 96, 24]),
    (512, 128, [40, 20, 16]),
    (320, 96, [36, 28, 32]),
    (544, 256, [136, 260, 100, 44]),
    (1024, 512, [384, 128, 256]),
    (96, 32, [12, 24]),
]


@pytest.mark.parametrize("dt", ["int8", "bf16"])
@pytest.mark.parametrize("shape", CHAIN_SHAPES)
def test_chain_matches_oracle_ref_semantics(fg, dt, shape):
    N, K1, Ms = shape
    B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=len(Ms) * 1000 + N)
    want = oracle.chain(dt, B, As, N, Ms, Ks, mode=oracle.REF, threads=1)
    got = run_chain(fg, dt, B, As, N, Ms, Ks)
    rows = (Ms[-1] // 4) * 4 if dt == "int8" else None
    assert_parity(dt, got, want, rows)


@pytest.mark.parametrize("dt", ["int8", "bf16"])
@pytest.mark.parametrize("shape", CHAIN_SHAPES[:4])
def test_chain_math_semantics(fg, dt, shape):
    N, K1, Ms = shape
    B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=7 + N)
    fg.set_semantics("math")
    try:
        got = run_chain(fg, dt, B, As, N, Ms, Ks)
    finally:
        fg.set_semantics("ref")
    want = oracle.chain(dt, B, As, N, Ms, Ks, mode=oracle.MATH)
    assert_parity(dt, got, want)
    if dt == "bf16":
        Bf = oracle.bf16_to_f32(B)
        Af = [oracle.bf16_to_f32(a) for a in As]
        assert oracle.rel_frob(got, oracle.chain_f64(Bf, Af, N, Ms, Ks)) < BF16_VS_FP64


@pytest.mark.parametrize("shape", [(256, 64, [48, 96, 24]), (520, 100, [130, 66]),
                                   (100, 64, [40, 24])])
def test_f32_chain_ffma_bitexact_and_3xtf32_accuracy(fg, shape):
    N, K1, Ms = shape
    B, As, Ks = oracle.chain_inputs("f32", N, K1, Ms, seed=N)
    want32 = oracle.chain("f32", B, As, N, Ms, Ks)
    want64 = oracle.chain_f64(B, As, N, Ms, Ks)
    fg.set_f32_algo("ffma")
    try:
        ffma = run_chain(fg, "f32", B, As, N, Ms, Ks)
    finally:
        fg.set_f32_algo("3xtf32")
    np.testing.assert_array_equal(ffma, want32)
    tf = run_chain(fg, "f32", B, As, N, Ms, Ks)
    e_ffma = oracle.rel_frob(ffma, want64)
    e_tf = oracle.rel_frob(tf, want64)
    assert e_tf <= 2 * e_ffma, (e_tf, e_ffma)


@pytest.mark.parametrize("shape", [(1024, 1024, 1024), (128, 2048, 4096), (512, 64, 128),
                                   (777, 333, 129)])
def test_sgemm_ffma_bitexact_and_3xtf32(fg, shape):
    M, N, K = shape
    A, B = oracle.sgemm_inputs(M, N, K, seed=M)
    want = oracle.sgemm_f32(A, B, kblock=2048)
    C = np.zeros((M, N), np.float32)
    fg.LibShalom_sgemm_mp(0, 0, C, A, B, M, N, K, check=True)
    np.testing.assert_array_equal(C, want)
    want64 = oracle.sgemm_f64(A, B)
    fg.set_sgemm_algo("3xtf32")
    try:
        C2 = np.zeros((M, N), np.float32)
        fg.LibShalom_sgemm_mp(0, 0, C2, A, B, M, N, K, check=True)
    finally:
        fg.set_sgemm_algo("ffma")
    assert oracle.rel_frob(C2, want64) <= 2 * oracle.rel_frob(C, want64)


def test_sgemm_nt_mode_leaves_c_untouched(fg):
    A, B = oracle.sgemm_inputs(64, 64, 64, seed=1)
    C = np.full((64, 64), 3.0, np.float32)
    fg.LibShalom_sgemm_mp(0, 1, C, A, B, 64, 64, 64, check=True)
    assert (C == 3.0).all()


# ---------------------------------------------------------------- full sizes (sampled panels)

def _panel_cols(N, panels):
    return np.concatenate([np.arange(32 * p, 32 * p + 32) for p in panels])


@pytest.mark.parametrize("dt,N,K1,Ms", [
    ("bf16", 4096, 1024, [4096, 1024, 1024]),             # BF16 chain of 3 GEMMs
    ("int8", 8192, 2048, [4096, 2048, 4096, 1024]),       # INT8 chain of 4 GEMMs
])
def test_full_size_chain_on_sampled_panels(fg, dt, N, K1, Ms):
    """The reference's permutation stays inside 32-column panels, so panel p of C
    depends only on panel p of B: full-size results are checked exactly on a
    sample of panels by running the oracle on just those columns."""
    B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=2024)
    got = run_chain(fg, dt, B, As, N, Ms, Ks)
    panels = [0, 1, N // 64, N // 32 - 1]
    cols = _panel_cols(N, panels)
    Bs = np.ascontiguousarray(B[:, cols])
    want = oracle.chain(dt, Bs, As, len(cols), Ms, Ks, mode=oracle.REF, threads=1)
    rows = (Ms[-1] // 4) * 4 if dt == "int8" else None
    assert_parity(dt, np.ascontiguousarray(got[:, cols]), want, rows)
    if dt == "int8":
        # every stage saturates at these widths: the output is bounded by K * 255 * 128
        assert np.abs(got.astype(np.int64)).max() <= Ks[-1] * 255 * 128


# ---------------------------------------------------------------- device entry points

@pytest.mark.parametrize("dt", ["int8", "bf16", "f32"])
def test_device_api_matches_host_api(fg, dt):
    import torch
    N, K1, Ms = 512, 128, [256, 96, 64]
    B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=99)
    host = run_chain(fg, dt, B, As, N, Ms, Ks)
    tdt = {"int8": torch.int8, "bf16": torch.int16, "f32": torch.float32}[dt]
    tB = torch.from_numpy(B.view(np.int8) if dt == "int8" else
                          (B.view(np.int16) if dt == "bf16" else B)).cuda()
    tA = [torch.from_numpy(a.view(np.int16) if dt == "bf16" else a).cuda() for a in As]
    tC = torch.zeros((Ms[-1], N), dtype=torch.int32 if dt == "int8" else torch.float32,
                     device="cuda")
    fg.chain_dev(dt, tC, tB, N, tA, Ms, Ks)
    torch.cuda.synchronize()
    fg.sync()
    np.testing.assert_array_equal(tC.cpu().numpy(), host)
    assert tdt is not None


def test_odd_k_prints_and_returns_like_the_reference(fg, capfd):
    B, As, Ks = oracle.chain_inputs("f32", 64, 63, [32], seed=1)
    C = np.full((32, 64), 7.0, np.float32)
    fg.flashgemm_multi_f32f32f32(C, B, 64, 1, As[0], 32, 63)
    assert "K must be a multiple of 2" in capfd.readouterr().out
    assert fg.last_status() == fg.FG_ERR_INVALID
    assert (C == 7.0).all()


def test_mismatched_chain_is_rejected(fg):
    B, As, Ks = oracle.chain_inputs("int8", 64, 64, [32, 32], seed=1)
    C = np.zeros((32, 64), np.int32)
    fg.flashgemm_multi_int8uint8int32(C, B, 64, 2, As[0], 32, 64, As[1], 32, 48)
    assert fg.last_status() == fg.FG_ERR_INVALID


@pytest.mark.parametrize("dt", ["int8", "bf16"])
def test_fused_chain_equals_per_gemm_path(fg, dt):
    """One persistent launch for the whole chain computes exactly what one
    launch per GEMM computes (same tiles, same k order)."""
    N, K1, Ms = 1280, 256, [384, 520, 136, 64]
    B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=31)
    fg.set_chain_mode("per_gemm")
    try:
        a = run_chain(fg, dt, B, As, N, Ms, Ks)
    finally:
        fg.set_chain_mode("fused")
    b = run_chain(fg, dt, B, As, N, Ms, Ks)
    np.testing.assert_array_equal(a, b)
    want = oracle.chain(dt, B, As, N, Ms, Ks, mode=oracle.REF, threads=1)
    assert_parity(dt, b, want, (Ms[-1] // 4) * 4 if dt == "int8" else None)


_STREAM_SCRIPT = """
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import flashgemm_b200 as fg, oracle
dt, out = sys.argv[2], sys.argv[3]
N, K1, Ms = 768, 256, [1000, 520, 136, 300]
B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=43)
fg.set_semantics("ref")
C = np.zeros((Ms[-1], N), np.int32 if dt == "int8" else np.float32)
args = []
for a, m, k in zip(As, Ms, Ks):
    args += [a, m, k]
getattr(fg, {"int8": "flashgemm_multi_int8uint8int32",
             "bf16": "flashgemm_multi_bf16bf16f32"}[dt])(C, B, N, len(Ms), *args, check=True)
fg.sync()
np.save(out, C)
"""


@pytest.mark.parametrize("dt", ["int8", "bf16"])
def test_streamed_hand_off_is_bit_identical(dt, tmp_path):
    """The streamed hand-off between stages (a stage's tile waits for each
    256-row tile of its input as its k-loop reaches it) changes only when tiles
    start, not their arithmetic: forced on and forced off, the fused chain gives
    identical bits, here with stage K not a multiple of 256 and INT8 tail rows."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = {}
    for mode in ("0", "1"):
        path = str(tmp_path / f"c{mode}.npy")
        env = dict(os.environ, FG_CHAIN_STREAM=mode,
                   PYTHONPATH=os.pathsep.join([root, os.path.join(root, "oracle")]))
        r = subprocess.run([sys.executable, "-c", _STREAM_SCRIPT, root, dt, path], env=env,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        outs[mode] = np.load(path)
    np.testing.assert_array_equal(outs["0"], outs["1"])
    N, K1, Ms = 768, 256, [1000, 520, 136, 300]
    B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=43)
    want = oracle.chain(dt, B, As, N, Ms, Ks, mode=oracle.REF, threads=1)
    assert_parity(dt, outs["1"], want, (Ms[-1] // 4) * 4 if dt == "int8" else None)


_PARAMS_SCRIPT = """
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import flashgemm_b200 as fg, oracle
dt, out, N, K1 = sys.argv[2], sys.argv[3], int(sys.argv[4]), int(sys.argv[5])
Ms = [int(m) for m in sys.argv[6].split(",")]
B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=47)
fg.set_semantics("ref")
C = np.zeros((Ms[-1], N), np.int32 if dt == "int8" else np.float32)
args = []
for a, m, k in zip(As, Ms, Ks):
    args += [a, m, k]
getattr(fg, {"int8": "flashgemm_multi_int8uint8int32",
             "bf16": "flashgemm_multi_bf16bf16f32"}[dt])(C, B, N, len(Ms), *args, check=True)
fg.sync()
np.save(out, C)
"""


@pytest.mark.parametrize("dt,N,K1,Ms", [
    ("bf16", 1024, 256, [512, 288, 512]),                       # 3 stages, few entries
    ("int8", 768, 256, [520, 300, 264, 512, 280, 136]),         # 6 stages
])
def test_fused_chain_parameter_blocks_are_bit_identical(tmp_path, dt, N, K1, Ms):
    """A fused chain launched with the largest parameter block (FG_CHAIN_PARAMS=big)
    and with the smallest one its stages and schedule fit computes identical bits."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = {}
    for mode in ("", "big"):
        path = str(tmp_path / f"c{mode or 'default'}.npy")
        env = dict(os.environ, PYTHONPATH=os.pathsep.join([root, os.path.join(root, "oracle")]))
        env.pop("FG_CHAIN_PARAMS", None)
        if mode:
            env["FG_CHAIN_PARAMS"] = mode
        r = subprocess.run([sys.executable, "-c", _PARAMS_SCRIPT, root, dt, path, str(N), str(K1),
                            ",".join(map(str, Ms))], env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        outs[mode] = np.load(path)
    np.testing.assert_array_equal(outs[""], outs["big"])
    B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=47)
    want = oracle.chain(dt, B, As, N, Ms, Ks, mode=oracle.REF, threads=1)
    assert_parity(dt, outs[""], want, (Ms[-1] // 4) * 4 if dt == "int8" else None)


def test_int8_intermediates_l2_policy_is_bit_identical(tmp_path):
    """INT8 intermediates stored with an L2 evict-last policy (the default), with
    plain stores (FG_L2_KEEP=0), and with an L2 set-aside for them (FG_L2_KEEP=96)
    give identical bits: the policy only decides which lines stay in L2."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = {}
    for mode in ("", "0", "96"):
        path = str(tmp_path / f"c{mode or 'default'}.npy")
        env = dict(os.environ, PYTHONPATH=os.pathsep.join([root, os.path.join(root, "oracle")]))
        env.pop("FG_L2_KEEP", None)
        if mode:
            env["FG_L2_KEEP"] = mode
        r = subprocess.run([sys.executable, "-c", _STREAM_SCRIPT, root, "int8", path], env=env,
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        outs[mode] = np.load(path)
    np.testing.assert_array_equal(outs[""], outs["0"])
    np.testing.assert_array_equal(outs[""], outs["96"])
    N, K1, Ms = 768, 256, [1000, 520, 136, 300]
    B, As, Ks = oracle.chain_inputs("int8", N, K1, Ms, seed=43)
    want = oracle.chain("int8", B, As, N, Ms, Ks, mode=oracle.REF, threads=1)
    assert_parity("int8", outs[""], want, (Ms[-1] // 4) * 4)


@pytest.mark.parametrize("dt,f32algo", [("int8", None), ("bf16", None), ("f32", "ffma"),
                                        ("f32", "3xtf32")])
def test_registered_weights_match_per_call_weights(fg, dt, f32algo):
    """Weights registered once (copied, TF32-split / INT8 tail rows prepared)
    give exactly the per-call entry point's results, call after call."""
    import torch
    N, K1, Ms = 768, 200, [268, 1000, 44]   # INT8 tail rows in every stage, one past row 256
    if dt == "f32":
        fg.set_f32_algo(f32algo)
    try:
        B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=41)
        if dt == "int8":
            K1, Ks = 256, [256] + Ms[:-1]
            B, As, _ = oracle.chain_inputs(dt, N, K1, Ms, seed=41)
        host = run_chain(fg, dt, B, As, N, Ms, Ks)
        W = [fg.Weights(dt, a) for a in As]
        assert all(w.nbytes > 0 for w in W)
        tB = torch.from_numpy(B.view(np.int8) if dt == "int8" else
                              (B.view(np.int16) if dt == "bf16" else B)).cuda()
        for _ in range(2):
            tC = torch.zeros((Ms[-1], N), dtype=torch.int32 if dt == "int8" else torch.float32,
                             device="cuda")
            fg.chain_registered(dt, tC, tB, N, W)
            torch.cuda.synchronize()
            fg.sync()
            np.testing.assert_array_equal(tC.cpu().numpy(), host)
        for w in W:
            w.release()
    finally:
        fg.set_f32_algo("3xtf32")


@pytest.mark.parametrize("dt", ["int8", "bf16"])
def test_grouped_launch_matches_chains_run_alone(fg, dt):
    """Chains of uneven lengths and shapes in one grouped launch (more stages
    than fit in the kernel parameters, so the tables go through device memory)
    give exactly what each chain gives on its own."""
    import torch
    rng = np.random.default_rng(5)
    specs = []
    for j in range(7):
        n = int(rng.integers(2, 5))
        N = int(rng.choice([256, 512, 768, 1280]))
        dims = [int(rng.choice([64, 128, 272, 520, 1024]))] + \
               [int(rng.choice([128, 260, 384, 1000])) for _ in range(n)]
        if dt == "int8":
            dims[0] = max(64, dims[0] // 32 * 32)
        specs.append((N, dims[0], dims[1:]))
    chains, alone = [], []
    for j, (N, K1, Ms) in enumerate(specs):
        B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=100 + j)
        W = [fg.Weights(dt, a) for a in As]
        tB = torch.from_numpy(B.view(np.int8) if dt == "int8" else B.view(np.int16)).cuda()
        mk = lambda: torch.zeros((Ms[-1], N), dtype=torch.int32 if dt == "int8" else torch.float32,
                                 device="cuda")
        c1, c2 = mk(), mk()
        fg.chain_registered(dt, c1, tB, N, W)
        chains.append((c2, tB, N, W))
        alone.append(c1)
    fg.chain_group(dt, chains)
    torch.cuda.synchronize()
    fg.sync()
    for (c2, _, _, W), c1 in zip(chains, alone):
        np.testing.assert_array_equal(c2.cpu().numpy(), c1.cpu().numpy())
        for w in W:
            w.release()


# ---------------------------------------------------------------- one chain split across devices

@pytest.mark.parametrize("dt", ["int8", "bf16", "f32"])
@pytest.mark.parametrize("parts", [1, 3])
def test_chain_split_across_devices_equals_one_device(fg, dt, parts):
    """fg_chain_multi_device cuts the columns on 32-column panel boundaries and
    runs the unchanged chain on every slice; listing device 0 several times
    runs the parts one after another on this GPU. The result equals the
    single-call result bit for bit."""
    N, K1, Ms = 1312, 256, [384, 136, 100]
    B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=55)
    one = run_chain(fg, dt, B, As, N, Ms, Ks)
    C = np.zeros_like(one)
    fg.chain_multi_device(dt, C, B, N, As, Ms, Ks, devices=[0] * parts)
    rows = (Ms[-1] // 4) * 4 if dt == "int8" else Ms[-1]
    np.testing.assert_array_equal(C[:rows], one[:rows])
    if dt != "f32":
        assert_parity(dt, C, oracle.chain(dt, B, As, N, Ms, Ks, mode=oracle.REF, threads=1), rows)


@pytest.mark.parametrize("dt", ["int8", "bf16"])
def test_pinned_and_pageable_host_buffers_give_the_same_result(fg, dt):
    """Host operands in page-locked memory are copied directly; ordinary
    (pageable) ones pass through the library's pinned staging, chunk by chunk.
    Both, and a mix of the two, give the same result."""
    import torch
    N, K1, Ms = 2080, 256, [512, 136, 100]   # chunked (N >= 1024), last chunk narrower
    B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=66)
    pageable = run_chain(fg, dt, B, As, N, Ms, Ks)
    def pin(a):
        a = np.ascontiguousarray(a)
        v = a.view(np.int16) if a.dtype == np.uint16 else a
        return torch.from_numpy(v).pin_memory().numpy().view(a.dtype)
    odt = np.int32 if dt == "int8" else np.float32
    for pb, pa, pc in [(True, True, True), (True, False, False), (False, True, True)]:
        Bx = pin(B) if pb else B
        Ax = [pin(a) for a in As] if pa else As
        Cx = pin(np.zeros((Ms[-1], N), odt)) if pc else np.zeros((Ms[-1], N), odt)
        got = run_chain(fg, dt, Bx, Ax, N, Ms, Ks, C=Cx)
        np.testing.assert_array_equal(got, pageable)
