"""The serving loop: chain requests admitted by device memory, batched into
grouped launches while other batches are on the GPU.

Each request's result must be the one the same request gives alone through
fg_chain_registered (INT8 bit-exact; BF16 and FP32 with the same kernels give
the same bits, and the check allows the BF16 / 3xTF32 tolerances of the other
tests should a different kernel choice ever differ in rounding), whether it
ran in a mix of dtypes and shapes or by itself.
"""
import random
import threading
import time

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


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


def _weight_sets(fg, seed):
    rng = np.random.default_rng(seed)
    sets = []
    for j, dt in enumerate(["bf16", "int8", "f32", "bf16", "int8", "f32", "bf16"]):
        n = int(rng.integers(2, 5))
        K1 = int(rng.choice([64, 128, 256, 512]))
        Ms = [int(rng.choice([64, 96, 200, 256, 520])) for _ in range(n)]
        _, As, Ks = oracle.chain_inputs(dt, 64, K1, Ms, seed=seed + j)
        sets.append((dt, K1, Ms, [fg.Weights(dt, a) for a in As], As))
    return sets


def _release(sets):
    for st in sets:
        for w in st[3]:
            w.release()


def _oracle_check(fg, dt, As, B, got, N, Ms):
    """The request's result against the oracle: INT8 bit-exact (written rows),
    BF16 within the parity tolerance of the reference semantics, FP32 (3xTF32)
    within 2x the plain FP32 kernel's own error against FP64."""
    Ks = [As[0].shape[1]] + list(Ms[:-1])
    if dt == "int8":
        want = oracle.chain(dt, B.view(np.uint8), As, N, Ms, Ks, mode=oracle.REF, threads=1)
        rows = (Ms[-1] // 4) * 4
        np.testing.assert_array_equal(got[:rows], want[:rows])
    elif dt == "bf16":
        want = oracle.chain(dt, B, As, N, Ms, Ks, mode=oracle.REF, threads=1)
        assert oracle.rel_frob(got, want) <= 2e-3
    else:
        exact = oracle.chain_f64(B, As, N, Ms, Ks)
        plain = oracle.chain("f32", B, As, N, Ms, Ks)
        assert oracle.rel_frob(got, exact) <= 2 * oracle.rel_frob(plain, exact)


def _inputs(dt, K1, N, seed):
    rng = np.random.default_rng(seed)
    if dt == "int8":
        return rng.integers(-127, 128, size=(K1, N)).astype(np.int8)
    if dt == "bf16":
        return oracle.bf16_rne(rng.standard_normal((K1, N)).astype(np.float32))
    return rng.standard_normal((K1, N)).astype(np.float32)


def _alone(fg, dt, W, B, N, Mlast):
    import torch
    tB = torch.from_numpy(B.view(np.int16) if B.dtype == np.uint16 else B).cuda()
    C = torch.zeros((Mlast, N), dtype=torch.int32 if dt == "int8" else torch.float32,
                    device="cuda")
    fg.chain_registered(dt, C, tB, N, W)
    torch.cuda.synchronize()
    return C.cpu().numpy()


def _same(dt, got, want, Mlast):
    rows = (Mlast // 4) * 4 if dt == "int8" else Mlast
    if dt == "int8" or np.array_equal(got[:rows], want[:rows]):
        np.testing.assert_array_equal(got[:rows], want[:rows])
    else:
        tol = 1e-2 if dt == "bf16" else 1e-6
        assert oracle.rel_frob(got[:rows], want[:rows]) <= tol


def test_results_same_alone_and_in_the_mix(fg):
    """Requests of three dtypes and many shapes arrive at random times from two
    threads while earlier batches run; host and device buffers mixed."""
    import torch
    sets = _weight_sets(fg, 70)
    srv = fg.Server(max_batch=8, slots=2, max_wait_us=300)
    reqs = []
    lock = threading.Lock()

    def client(k):
        rnd = random.Random(k)
        for i in range(24):
            dt, K1, Ms, W, As = sets[rnd.randrange(len(sets))]
            N = rnd.choice([16, 64, 128, 272, 512])
            B = _inputs(dt, K1, N, 1000 * k + i)
            odt = np.int32 if dt == "int8" else np.float32
            if i % 3 == 2:  # device-resident request
                tB = torch.from_numpy(B.view(np.int16) if B.dtype == np.uint16 else B).cuda()
                C = torch.full((Ms[-1], N), 9, dtype=torch.int32 if dt == "int8" else torch.float32,
                               device="cuda")
                torch.cuda.synchronize()
                rid = srv.submit(dt, W, tB, C)
            else:
                C = np.full((Ms[-1], N), 9, odt)
                rid = srv.submit(dt, W, B, C)
            with lock:
                reqs.append((rid, dt, W, B, C, N, Ms, As))
            time.sleep(rnd.expovariate(4000.0))

    th = [threading.Thread(target=client, args=(k,)) for k in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    lats = [srv.wait(r[0]) for r in reqs]
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["batches"] < len(reqs)  # arrivals were batched
    assert st["p99_us"] >= st["p50_us"] > 0 and all(x > 0 for x in lats)
    for k, (rid, dt, W, B, C, N, Ms, As) in enumerate(reqs):
        got = C.cpu().numpy() if not isinstance(C, np.ndarray) else C
        _same(dt, got, _alone(fg, dt, W, B, N, Ms[-1]), Ms[-1])
        if k % 4 == 0:  # a sample of the mix, against the oracle directly
            _oracle_check(fg, dt, As, B, got, N, Ms)
    srv.close()
    _release(sets)


def test_admission_by_device_memory(fg):
    """With a budget that holds about one request, requests still all complete
    (admitted as memory frees up), the held bytes never exceed the budget, and
    a request larger than the whole budget fails alone without stalling the rest."""
    sets = _weight_sets(fg, 80)
    dt, K1, Ms, W, _ = sets[0]
    N = 256
    budget = 3 << 20
    srv = fg.Server(hbm_budget=budget, max_batch=16, slots=2)
    ids = []
    outs = []
    for i in range(12):
        B = _inputs(dt, K1, N, 2000 + i)
        C = np.zeros((Ms[-1], N), np.float32)
        ids.append(srv.submit(dt, W, B, C))
        outs.append((B, C))
    big_B = _inputs(dt, K1, 65536, 3000)
    big_C = np.zeros((Ms[-1], 65536), np.float32)
    big = srv.submit(dt, W, big_B, big_C)
    for rid in ids:
        srv.wait(rid)
    with pytest.raises(fg.FlashgemmError):
        srv.wait(big)
    st = srv.stats()
    assert st["completed"] == 12 and st["failed"] == 1
    assert 0 < st["peak_bytes"] <= budget
    for B, C in outs:
        _same(dt, C, _alone(fg, dt, W, B, N, Ms[-1]), Ms[-1])
    srv.close()
    _release(sets)


def test_burst_is_batched_and_stats_reset(fg):
    sets = _weight_sets(fg, 90)
    dt, K1, Ms, W, _ = sets[1]
    srv = fg.Server(max_batch=32, slots=2)
    B = _inputs(dt, K1, 128, 4000)
    Cs = [np.zeros((Ms[-1], 128), np.int32) for _ in range(96)]
    ids = [srv.submit(dt, W, B, C) for C in Cs]
    srv.drain()
    st = srv.stats()
    assert st["completed"] == 96 and st["batches"] <= 48 and st["mean_batch"] >= 2
    assert st["flops"] > 0 and st["span_s"] > 0
    for rid in ids:
        srv.wait(rid)
    want = _alone(fg, dt, W, B, 128, Ms[-1])
    for C in Cs:
        _same(dt, C, want, Ms[-1])
    srv.reset_stats()
    st = srv.stats()
    assert st["completed"] == 0 and st["batches"] == 0
    srv.close()
    _release(sets)


def test_load_shedding_bounds_queueing(fg):
    """A burst far above what the loop can admit within max_queue_us: the
    requests still queued at their deadline are shed (FG_ERR_BUSY, outputs
    untouched), every other request completes with the right result, and the
    counts add up."""
    sets = _weight_sets(fg, 95)
    dt, K1, Ms, W, As = sets[0]
    N = 512
    srv = fg.Server(max_batch=4, slots=1, max_queue_us=300)
    B = _inputs(dt, K1, N, 5000)
    Cs = [np.full((Ms[-1], N), 7.0, np.float32) for _ in range(200)]
    ids = [srv.submit(dt, W, B, C) for C in Cs]
    srv.drain()
    st = srv.stats()
    assert st["shed"] > 0 and st["completed"] > 0 and st["failed"] == 0
    assert st["completed"] + st["shed"] == 200
    want = _alone(fg, dt, W, B, N, Ms[-1])
    served = 0
    for rid, C in zip(ids, Cs):
        lat = srv.wait(rid, shed_ok=True)
        if lat is None:
            assert (C == 7.0).all()  # never run
            continue
        served += 1
        _same(dt, C, want, Ms[-1])
    assert served == st["completed"]
    _oracle_check(fg, dt, As, B, want, N, Ms)
    srv.close()
    _release(sets)
