"""fg_chain_bf16_noalloc: the BF16 chain for callers that cannot allocate device
memory when they run it (a framework that owns all device memory through its
own pool, a server that must not grow after start-up). Its between-stage
buffers live in a fixed array inside the library instead of memory obtained
with cudaMalloc, so these tests check that it computes exactly what the
allocating entry point (fg_chain_dev) computes, call after call, that both
agree with the oracle, that a status word the caller passes stays clear, and
that it refuses a chain whose intermediates do not fit in that array.

Collected last on purpose (file name), so that a run stopping at the first
failure has already run every other test."""
import ctypes

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

BF16_TOL = 2e-3  # the BF16 tolerance of the parity tests (against the reference semantics)


@pytest.fixture(scope="module")
def fg():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import flashgemm_b200 as fg
    L = fg.lib()
    f = L.fg_chain_bf16_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_void_p]
    fg.set_semantics("ref")
    fg.flashgemm_set_thread_num(1)
    return fg


def _device_operands(N, K1, Ms, seed):
    import torch
    B, As, Ks = oracle.chain_inputs("bf16", N, K1, Ms, seed=seed)
    tB = torch.from_numpy(B.view(np.int16)).cuda()
    tA = [torch.from_numpy(a.view(np.int16)).cuda() for a in As]
    return B, As, tB, tA, Ks


def _noalloc(fg, tC, tB, N, tA, Ms, Ks, status=None, stream=None):
    import torch
    n = len(tA)
    aptr = (ctypes.c_void_p * n)(*[a.data_ptr() for a in tA])
    ms = (ctypes.c_long * n)(*Ms)
    ks = (ctypes.c_long * n)(*Ks)
    s = (stream or torch.cuda.current_stream()).cuda_stream
    return fg.lib().fg_chain_bf16_noalloc(tC.data_ptr(), tB.data_ptr(), N, n, aptr, ms, ks,
                                          status, s)


@pytest.mark.parametrize("N,K1,Ms", [
    (512, 256, [384, 128, 96]),     # row stride = N
    (520, 136, [264, 104, 40]),     # N % 16 == 8: between-stage rows padded to 528 columns
])
def test_noalloc_matches_allocating_entry_point_on_consecutive_calls(fg, N, K1, Ms):
    import torch
    runs = []
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    for j, seed in enumerate((11, 12)):  # two calls in a row, different inputs, shared scratch
        B, As, tB, tA, Ks = _device_operands(N, K1, Ms, seed + N)
        tC = torch.full((Ms[-1], N), float("nan"), device="cuda")
        # first call: the caller's status word; second: the array's own word
        st = _noalloc(fg, tC, tB, N, tA, Ms, Ks, status=status.data_ptr() if j == 0 else None)
        assert st == fg.FG_OK, fg.last_error()
        runs.append((B, As, tB, tA, Ks, tC))
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    fg.sync()  # reports a time-out of the status == NULL call, if there was one
    for B, As, tB, tA, Ks, tC in runs:
        ref = torch.zeros((Ms[-1], N), device="cuda")
        fg.chain_dev("bf16", ref, tB, N, tA, Ms, Ks)
        torch.cuda.synchronize()
        fg.sync()
        got, want = tC.cpu().numpy(), ref.cpu().numpy()
        # every kernel choice computes the same per-element products in the same order
        np.testing.assert_array_equal(got, want)
        exact = oracle.chain("bf16", B, As, N, Ms, Ks, mode=oracle.REF, threads=1)
        assert oracle.rel_frob(got, exact) <= BF16_TOL


def test_noalloc_rejects_chain_larger_than_its_scratch(fg):
    import torch
    N, Ms, Ks = 8192, [4096, 4096, 64], [64, 4096, 4096]
    tB = torch.zeros((Ks[0], N), dtype=torch.int16, device="cuda")
    tA = [torch.zeros((m, k), dtype=torch.int16, device="cuda") for m, k in zip(Ms, Ks)]
    tC = torch.zeros((Ms[-1], N), device="cuda")
    st = _noalloc(fg, tC, tB, N, tA, Ms, Ks)
    assert st == fg.FG_ERR_INVALID
    assert "FG_NOALLOC_SCRATCH_BYTES" in fg.last_error()
