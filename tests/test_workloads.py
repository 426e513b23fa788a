"""The benchmark's synthetic workloads have the shapes and mixes they are stated
to have (host only, no GPU): the grouped FP32 chains and the serving stream."""
import math
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_group_specs_shapes():
    specs = bench.group_specs(4321)
    assert len(specs) == bench.GROUP_CHAINS
    thin = [s for s in specs if s[0] == 65536]
    assert len(thin) == bench.GROUP_SKINNY
    for N, K1, Ms in thin:
        assert K1 == 64 and all(m == 64 for m in Ms) and 2 <= len(Ms) <= 5
    dims, cols = [], []
    for N, K1, Ms in specs:
        if N == 65536:
            continue
        assert 2 <= len(Ms) <= 5
        for d in [K1] + Ms:
            assert 64 <= d <= 4096 and d % 16 == 0
            dims.append(d)
        assert 64 <= N <= 8192 and N % 16 == 0
        cols.append(N)
    # log-uniform: the median sits near the geometric mean of the range
    assert abs(math.log(np.median(dims)) - math.log(512)) < 0.35
    assert abs(math.log(np.median(cols)) - math.log(math.sqrt(64 * 8192))) < 0.35
    # the same seed gives the same workload
    assert bench.group_specs(4321) == specs


def test_group_sample_is_bounded_and_includes_skinny():
    specs = bench.group_specs(4321)
    sample = bench.group_sample(specs, 4322)
    assert len(sample) == len(set(sample)) >= 10
    assert sum(1 for i in sample if specs[i][0] == 65536) == 2
    assert all(bench.flops_of(*specs[i]) <= 20e9 for i in sample if specs[i][0] != 65536)
    only_thin = bench.group_specs(1, count=8, skinny=8)
    assert all(s[0] == 65536 for s in only_thin)
    assert bench.group_sample(only_thin, 2)  # no regular chains: the skinny ones only


def test_serve_sets_and_requests():
    sets = bench.serve_sets(777)
    assert len(sets) == bench.SERVE_SETS
    counts = {d: sum(1 for s in sets if s[0] == d) for d in ("bf16", "int8", "f32")}
    assert counts == {"bf16": 32, "int8": 19, "f32": 13}
    for dt, K1, Ms in sets:
        assert 2 <= len(Ms) <= 6
        assert all(64 <= d <= 4096 and d % 16 == 0 for d in [K1] + Ms)
    reqs = bench.serve_requests(787, sets, 20000)
    frac = {d: sum(1 for i, _ in reqs if sets[i][0] == d) / len(reqs) for d in ("bf16", "int8", "f32")}
    assert abs(frac["bf16"] - 0.5) < 0.02 and abs(frac["int8"] - 0.3) < 0.02
    assert abs(frac["f32"] - 0.2) < 0.02
    assert all(64 <= N <= 4096 and N % 16 == 0 for _, N in reqs)
