"""The CUDA path against the reference's own code (oracle/_ref: the
reference's src/shcoll/src compiled unmodified over emulated PEs), directly,
at the configured shapes: the 64-member x 2^20 headline in all three
butterfly orders, teams of 100-256 members (deep butterflies and large
extra-PE folds), and the 128-member data-movement shapes.  The restatement
is not in the loop here: a mistake shared by the kernels and the
restatement would still be caught."""
import numpy as np
import pytest

import gen
import oracle
from test_reduce_gpu import gpu_reduce, nan_equal_bytes

pytestmark = pytest.mark.gpu

TNAME = {np.dtype(np.float32): "float", np.dtype(np.float64): "double",
         np.dtype(np.int32): "int32", np.dtype(np.int64): "int64", np.dtype(np.uint64): "uint64"}


def ref_reduce(ref, algo, op, x):
    y, _ = ref.reduce(algo, op, x, tname=TNAME[x.dtype])
    return y


@pytest.mark.parametrize("op,dt,algo", [
    ("sum", np.float32, "rec_dbl"), ("sum", np.float32, "rabenseifner"),
    ("sum", np.float32, "rabenseifner2"), ("max", np.float64, "rec_dbl"),
    ("max", np.float64, "rabenseifner"), ("xor", np.int64, "rec_dbl"),
    ("xor", np.int64, "rabenseifner")])
def test_config2_full_size_matches_reference(B, heap, ref, op, dt, algo):
    """64 members x 2^20 elements with the configured distributions."""
    P, N = 64, 1 << 20
    if op == "sum":
        x = gen.normal(dt, P, N, 21)
    elif op == "max":
        x = gen.uniform(dt, P, N, 22, -1e6, 1e6)
    else:
        x = gen.uniform_int(dt, P, N, 23)
    got = gpu_reduce(B, heap, algo, op, x)
    assert got.tobytes() == ref_reduce(ref, algo, op, x).tobytes()


@pytest.mark.parametrize("P", [100, 128, 255, 256])
def test_large_teams_match_reference(B, heap, ref, P):
    """Float SUM/PROD trees over 100-256 members in every deterministic
    order, integer ops, and order-dependent MIN/MAX (NaN payloads, +-0)."""
    N = 2 * P + 37
    for dt in (np.float32, np.float64):
        s = gen.normal(dt, P, N, P)
        p = gen.uniform(dt, P, N, P + 1, 0.99, 1.01)
        mm = gen.special_minmax(dt, P, N, P + 2)
        for algo in ("rec_dbl", "rabenseifner", "rabenseifner2", "linear"):
            assert gpu_reduce(B, heap, algo, "sum", s).tobytes() == \
                ref_reduce(ref, algo, "sum", s).tobytes(), (dt, algo, "sum")
            assert gpu_reduce(B, heap, algo, "prod", p).tobytes() == \
                ref_reduce(ref, algo, "prod", p).tobytes(), (dt, algo, "prod")
            for op in ("min", "max"):
                assert gpu_reduce(B, heap, algo, op, mm).tobytes() == \
                    ref_reduce(ref, algo, op, mm).tobytes(), (dt, algo, op)
    xi = gen.uniform_int(np.int32, P, N, P + 3)
    for op in ("sum", "prod", "xor", "min"):
        assert gpu_reduce(B, heap, "rec_dbl", op, xi).tobytes() == \
            ref_reduce(ref, "rec_dbl", op, xi).tobytes(), op


def test_nan_sum_matches_reference_up_to_payload(B, heap, ref):
    """SUM over NaN inputs at 128 members: equal up to the NaN payload (x86
    carries payloads through +, the GPU gives the canonical NaN)."""
    x = gen.special_minmax(np.float64, 128, 300, 5)
    got = gpu_reduce(B, heap, "rec_dbl", "sum", x)
    assert nan_equal_bytes(got, ref_reduce(ref, "rec_dbl", "sum", x))


def test_config3_copies_match_reference(B, ref):
    """128 members: fcollect64 of 4096 int64, alltoallmem of 64 KiB blocks,
    alltoalls64 with dst 2 and sst 3 over 4096 elements per pair."""
    P = 128
    team = (0, 1, P)
    x = gen.uniform_int(np.int64, P, 4096, 31)
    want = np.zeros((P, P * 4096), np.int64)
    ref.run(oracle.K_SIZED, "shcoll_fcollect64_bruck_inplace", x, want, nelems=4096)
    src, dst = B.malloc(x[0].nbytes), B.malloc(want[0].nbytes)
    B.put_rows(src, x, team=team)
    B.fcollect(dst, src, x[0].nbytes, team=team)
    got = B.get_rows(dst, want[0].nbytes, np.int64, team=team)
    B.free(src)
    B.free(dst)
    assert got.tobytes() == want.tobytes()

    x = gen.uniform_int(np.uint8, P, P * 65536, 32)
    want = np.zeros_like(x)
    ref.run(oracle.K_TEAM_COPY, "shcoll_alltoallmem_shift_exchange_barrier", x, want,
            nelems=65536)
    src, dst = B.malloc(x[0].nbytes), B.malloc(x[0].nbytes)
    B.put_rows(src, x, team=team)
    B.alltoall(dst, src, 65536, team=team)
    got = B.get_rows(dst, x[0].nbytes, np.uint8, team=team)
    B.free(src)
    B.free(dst)
    assert got.tobytes() == want.tobytes()
    del x, want

    n = 4096
    x = gen.uniform_int(np.int64, P, P * n * 3, 33)
    d0 = gen.uniform_int(np.int64, P, P * n * 2, 34)
    want = d0.copy()
    ref.run(oracle.K_ALLTOALLS_SIZED, "shcoll_alltoalls64_shift_exchange_barrier", x, want,
            nelems=n, a=2, b=3)
    src, dst = B.malloc(x[0].nbytes), B.malloc(d0[0].nbytes)
    B.put_rows(src, x, team=team)
    B.put_rows(dst, d0, team=team)
    B.alltoalls(dst, src, 2, 3, n, 8, team=team)
    got = B.get_rows(dst, d0[0].nbytes, np.int64, team=team)
    B.free(src)
    B.free(dst)
    assert got.tobytes() == want.tobytes()
