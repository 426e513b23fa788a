"""The N > 1 path on CPU: two gloo ranks split one chain by activation
columns with the library's own partition (fg_split_columns, through
flashgemm_b200.shard_columns; host arithmetic that needs no GPU, the same one
fg_chain_multi_device and the column-partitioned bench ranks use), each
computes its slice with the reference semantics, and the gathered slices equal
the unsplit chain bit for bit. No data-path collective: the all_gather here
only assembles the answer for the check."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, dt, N, K1, Ms, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import flashgemm_b200 as fg
        B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=77)
        c0, c1 = fg.shard_columns(N, world, rank)
        Bs = np.ascontiguousarray(B[:, c0:c1])
        part = oracle.chain(dt, Bs, As, c1 - c0, Ms, Ks, mode=oracle.REF, threads=1)
        gathered = [None] * world
        dist.all_gather_object(gathered, ((c0, c1), part))
        if rank == 0:
            full = np.concatenate([g[1] for g in gathered], axis=1).astype(np.float64)
            q.put((full, [g[0] for g in gathered]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dt,N", [("int8", 320), ("bf16", 256), ("int8", 100)])
def test_column_sharding_matches_unsplit_chain(dt, N):
    K1, Ms = 64, [48, 96, 24]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, dt, N, K1, Ms, q))
             for r in range(world)]
    for p in procs:
        p.start()
    full, sizes = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed=77)
    want = oracle.chain(dt, B, As, N, Ms, Ks, mode=oracle.REF, threads=1)
    np.testing.assert_array_equal(full, want.astype(np.float64))
    assert sizes[0][0] == 0 and sizes[-1][1] == N
    assert all(a % 32 == 0 for a, _ in sizes)


def test_shard_columns_covers_range():
    import flashgemm_b200 as fg
    for N in [1, 31, 32, 100, 4096, 8192 + 16]:
        for w in [1, 2, 3, 8]:
            spans = [fg.shard_columns(N, w, r) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == N
            for (a, b), (c, d) in zip(spans, spans[1:]):
                assert b == c and a <= b
