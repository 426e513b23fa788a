"""Failure detection on the GPU, without a GPU fault.

Every wait in the library's kernels (pipeline barriers and the fused chain's
cross-CTA dependency counters) is bounded in time; a wait that runs out writes
an error code into a device status word, every warp leaves its loop, waits
(bounded) for its own copies and MMAs, frees tensor memory and returns, and the
host turns the code into FG_ERR_TIMEOUT. The reference has no such path (its
only error path is print-and-return, multigemm/src/flashgemm.c:64-68).

fg_selftest_timeout makes one wait run out on purpose: a fused chain whose
second stage waits on a dependency counter that nothing releases, with the
wait limit of that one launch lowered to a few milliseconds. Nothing traps,
faults or spins without a bound; these tests check that the time-out is
reported and that the next calls on the same context compute correctly.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fg():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import flashgemm_b200 as fg
    fg.lib()
    fg.set_semantics("ref")
    fg.flashgemm_set_thread_num(1)
    return fg


def _chain_ok(fg, dt, seed):
    N, K1, Ms = 512, 256, [384, 136, 96]
    B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=seed)
    C = np.zeros((Ms[-1], N), np.int32 if dt == "int8" else np.float32)
    trip = []
    for a, m, k in zip(As, Ms, Ks):
        trip += [a, m, k]
    fn = {"bf16": fg.flashgemm_multi_bf16bf16f32, "int8": fg.flashgemm_multi_int8uint8int32}[dt]
    fn(C, B, N, len(Ms), *trip, check=True)
    want = oracle.chain(dt, B, As, N, Ms, Ks, mode=oracle.REF, threads=1)
    if dt == "int8":
        np.testing.assert_array_equal(C, want)
    else:
        assert oracle.rel_frob(C, want) <= 2e-3


def test_stuck_dependency_times_out_and_is_reported(fg):
    import time
    t0 = time.perf_counter()
    st = fg.selftest_timeout(2000)  # 2 ms limit for that one launch
    dt = time.perf_counter() - t0
    assert st == fg.FG_ERR_TIMEOUT, (st, fg.last_error())
    assert "wait ran out" in fg.last_error()
    assert dt < 5.0  # the kernel returned on its own, long before the default 2 s limit
    fg.sync()  # the status word was cleared when it was read


def test_context_stays_usable_after_a_time_out(fg):
    for rep in range(2):
        assert fg.selftest_timeout(1000 + 1000 * rep) == fg.FG_ERR_TIMEOUT
        # the wait limit is back to its default: fused chains run to completion
        _chain_ok(fg, "bf16", seed=60 + rep)
        _chain_ok(fg, "int8", seed=70 + rep)
        fg.sync()


def test_selftest_rejects_out_of_range_limits(fg):
    assert fg.selftest_timeout(10) == fg.FG_ERR_INVALID
    assert fg.selftest_timeout(10 ** 7) == fg.FG_ERR_INVALID
