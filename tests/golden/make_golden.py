"""Generate the golden fixtures from the reference's own shcoll code.

Run in a checkout that has the reference tree (it builds oracle/_ref from
it):   python tests/golden/make_golden.py

Every output stored here was produced by the reference's unmodified
src/shcoll/src algorithms running over emulated PEs (oracle/ref_harness).
The fixtures pin the CPU restatement (oracle/shcoll_oracle.c) and the GPU
kernels wherever the reference tree is absent.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import oracle  # noqa: E402
import gen  # noqa: E402

TNAME = {"int32": "int32", "int64": "int64", "uint8": "uint8", "float32": "float",
         "float64": "double", "complex64": "complexf", "complex128": "complexd"}


def special_floats(dtype, P, N, seed):
    """Values that make float MIN/MAX order dependent: NaNs, +0 and -0."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((P, N)).astype(dtype)
    pick = rng.integers(0, 4, size=(P, N))
    x[pick == 0] = 0.0
    x[pick == 1] = -0.0
    nan_mask = rng.random((P, N)) < 0.15
    x[nan_mask] = np.nan
    if np.dtype(dtype) == np.float32:
        bits = x.view(np.uint32)
        bits[nan_mask] |= rng.integers(1, 1 << 22, size=nan_mask.sum(), dtype=np.uint32)
    else:
        bits = x.view(np.uint64)
        bits[nan_mask] |= rng.integers(1, 1 << 51, size=nan_mask.sum(), dtype=np.uint64)
    return x


def main():
    oracle.build(reference=True)
    R = oracle.Reference()
    out = {}

    # config 1: int32 sum_reduce (team WORLD, rec_dbl default), fcollect64
    # (active-set form, bruck_inplace default), barrier_all (binomial_tree)
    x, fc = gen.config1_inputs()
    y, _ = R.reduce("rec_dbl", "sum", x, tname="int32")
    fco = np.zeros((8, 8 * 256), np.int64)
    R.run(oracle.K_SIZED, "shcoll_fcollect64_bruck_inplace", fc, fco, nelems=256)
    R.run(oracle.K_BARRIER_ALL, "shcoll_barrier_all_binomial_tree", np.zeros((8, 1), np.int8),
          np.zeros((8, 1), np.int8))
    out["config1"] = dict(reduce_in=x, reduce_out=y, fcollect_in=fc, fcollect_out=fco)

    # reductions over every algorithm, a few dtypes, pow2 and non-pow2 teams
    cases = {}
    k = 0
    for algo in oracle.ALGOS:
        for dt, ops in [("int32", ["sum", "xor", "min"]), ("int64", ["prod", "and"]),
                        ("uint8", ["sum", "max"]), ("float32", ["sum", "prod", "max"]),
                        ("float64", ["sum", "min"]), ("complex128", ["sum", "prod"]),
                        ("complex64", ["prod"])]:
            if algo == "binomial" and dt.startswith(("float", "complex")):
                continue  # arrival-order dependent in the reference: no single answer
            for op in ops:
                for P, N in [(5, 13), (8, 11)]:
                    xin = gen.random_values(dt, P, N, 1000 + k)
                    yout, _ = R.reduce(algo, op, xin, tname=TNAME[dt])
                    cases[f"{algo}/{op}/{dt}/{P}"] = (xin, yout)
                    k += 1
    # order-dependent float MIN/MAX (NaN payloads, mixed-sign zeros)
    for algo in ["linear", "rec_dbl", "rabenseifner", "rabenseifner2"]:
        for dt in ["float32", "float64"]:
            for op in ["min", "max"]:
                for P, N in [(6, 16), (8, 9)]:
                    xin = special_floats(dt, P, N, 5000 + k)
                    yout, _ = R.reduce(algo, op, xin, tname=TNAME[dt])
                    cases[f"special/{algo}/{op}/{dt}/{P}"] = (xin, yout)
                    k += 1
    out["reduce"] = {}
    for name, (xin, yout) in cases.items():
        out["reduce"][name + "/in"] = xin
        out["reduce"][name + "/out"] = yout

    # data movement
    rng = np.random.default_rng(77)
    cp = {}
    x = rng.integers(0, 256, size=(5, 40), dtype=np.uint8)
    o = np.zeros((5, 200), np.uint8)
    R.run(oracle.K_TEAM_COPY, "shcoll_fcollectmem_bruck_inplace", x, o, nelems=40)
    cp["fcollect/in"], cp["fcollect/out"] = x, o.copy()
    x = rng.integers(0, 256, size=(6, 6 * 24), dtype=np.uint8)
    o = np.zeros_like(x)
    R.run(oracle.K_TEAM_COPY, "shcoll_alltoallmem_shift_exchange_barrier", x, o, nelems=24)
    cp["alltoall/in"], cp["alltoall/out"] = x, o.copy()
    n, dst, sst = 5, 2, 3
    x = rng.integers(-2**62, 2**62, size=(4, 4 * n * sst), dtype=np.int64)
    d0 = rng.integers(-9, 9, size=(4, 4 * n * dst), dtype=np.int64)
    o = d0.copy()
    R.run(oracle.K_ALLTOALLS_SIZED, "shcoll_alltoalls64_shift_exchange_barrier", x, o,
          nelems=n, a=dst, b=sst)
    cp["alltoalls/in"], cp["alltoalls/dest0"], cp["alltoalls/out"] = x, d0, o.copy()
    out["copy"] = cp

    manifest = {}
    for group, arrays in out.items():
        path = os.path.join(HERE, group + ".npz")
        np.savez_compressed(path, **arrays)
        manifest[group + ".npz"] = {k: hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest()
                                    for k, v in sorted(arrays.items())}
    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    print("wrote", ", ".join(sorted(manifest)))


if __name__ == "__main__":
    main()
