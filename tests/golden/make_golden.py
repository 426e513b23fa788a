"""Generate the golden vectors in this folder from the reference itself.

Runs the reference's own CPU implementation (compiled from its sources by
`make -C oracle ref` into oracle/_ref/) on seeded inputs and stores inputs and
outputs as .npz fixtures. Needs the reference sources, so it runs only where
they are mounted; the fixtures it writes are committed and are all the tests
need elsewhere.

    python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle  # noqa: E402

SENTINEL = 0x5A5A5A5A

# (name, dtype, N, K1, Ms, threads, seed, store_inputs)
CHAINS = [
    ("f32_chain_n96", "f32", 96, 64, [40, 24], 8, 11, True),
    ("bf16_chain_3stage", "bf16", 256, 64, [48, 96, 24], 8, 12, True),
    ("bf16_chain_tails", "bf16", 128, 96, [40, 20, 16], 1, 13, True),
    ("int8_chain_3stage", "int8", 256, 64, [48, 96, 24], 8, 14, True),
    ("int8_chain_tails", "int8", 128, 128, [40, 20, 16], 1, 15, True),
    ("int8_chain_c3_widths", "int8", 64, 256, [128, 64, 128, 32], 2, 16, True),
    ("int8_chain_unwritten_rows", "int8", 64, 64, [24, 18], 2, 17, True),
]
# (name, M, N, K, seed, store_inputs)
SGEMMS = [
    ("f32_sgemm_96x128x64", 96, 128, 64, 21, True),
    ("f32_sgemm_ksplit_48x128x2080", 48, 128, 2080, 22, False),
    ("f32_sgemm_mgn_768x64x96", 768, 64, 96, 23, False),
]


def sha(*arrs):
    h = hashlib.sha256()
    for a in arrs:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main():
    if not oracle.ref_available():
        sys.exit("oracle/_ref missing: run `make -C oracle ref` where the reference is mounted")
    for name, dt, N, K1, Ms, T, seed, store in CHAINS:
        B, As, Ks = oracle.chain_inputs(dt, N, K1, Ms, seed)
        C = np.zeros((Ms[-1], N), np.int32 if dt == "int8" else np.float32)
        if dt == "int8":
            C[:] = SENTINEL
        oracle.ref_chain(dt, B, As, N, Ms, Ks, threads=T, C=C)
        out = dict(dtype=dt, N=N, K1=K1, Ms=np.array(Ms), Ks=np.array(Ks), threads=T, seed=seed,
                   C=C, input_sha256=sha(B, *As), sentinel=SENTINEL)
        if store:
            out["B"] = B
            for i, a in enumerate(As):
                out[f"A{i}"] = a
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, C.shape)
    for name, M, N, K, seed, store in SGEMMS:
        A, B = oracle.sgemm_inputs(M, N, K, seed)
        C = oracle.ref_sgemm(A, B)
        out = dict(dtype="f32", M=M, N=N, K=K, seed=seed, C=C, input_sha256=sha(A, B))
        if store:
            out["A"] = A
            out["B"] = B
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, C.shape)


if __name__ == "__main__":
    main()
