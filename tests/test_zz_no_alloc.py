"""b200shm_reduce_noalloc: the all-reduce for callers that cannot allocate
device memory (their runtime owns every device allocation, or they may not
call cudaMalloc at all).  It takes the caller's device buffers and keeps
its only scratch -- the list of order-dependent float MIN/MAX elements -- in
a static device array, so it must give exactly what b200shm_reduce gives,
call after call, and must refuse sizes that array cannot hold.

This file is collected last on purpose: if it fails, a run that stops at
the first failure has already run every other test."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT = 1 << 18  # elements per member for float MIN/MAX (the static list)


def order_dependent(dtype, P, N, seed):
    """Inputs with NaNs and mixed-sign zeros, so the static list is used."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((P, N)).astype(dtype)
    pick = rng.integers(0, 6, size=(P, N))
    x[pick == 0] = 0.0
    x[pick == 1] = -0.0
    x[rng.random((P, N)) < 0.05] = np.nan
    return x


@pytest.mark.parametrize("op,dt,algo,P,N,in_place", [
    ("min", "float32", "rec_dbl", 8, 4099, False),
    ("max", "float64", "rabenseifner", 6, 1000, True),
    ("min", "float64", "linear", 64, 333, False),
    ("sum", "float32", "rec_dbl", 64, 1 << 16, False),
    ("xor", "int64", "binomial", 13, 777, False),
])
def test_noalloc_matches_b200shm_reduce_twice(B, heap, op, dt, algo, P, N, in_place):
    npdt = {"float32": np.float32, "float64": np.float64, "int64": np.int64}[dt]
    if dt.startswith("float"):
        x = order_dependent(npdt, P, N, P * 7 + N)
    else:
        x = np.random.default_rng(N).integers(-2**62, 2**62, size=(P, N), dtype=np.int64)
    team = (0, 1, P)
    nb = x[0].nbytes
    slice_bytes = B.lib.b200shm_heap_slice()
    src, ref = heap(nb), heap(nb)
    B.put_rows(src, x, team=team)
    B.reduce(op, dt, algo, ref, src, N, team=team)
    want = B.get_rows(ref, nb, npdt, team=team)
    for call in range(2):
        if in_place:
            dst = src
            B.put_rows(src, x, team=team)
        else:
            dst = heap(nb)
            B.memset(dst, 0xA5, nb, team=team)
        B.reduce_noalloc(op, dt, algo, P, B.ptr(0, dst), slice_bytes, B.ptr(0, src), slice_bytes, N)
        got = B.get_rows(dst, nb, npdt, team=team)
        assert got.tobytes() == want.tobytes(), f"call {call}"


def test_noalloc_rejects_sizes_beyond_its_static_list(B, heap):
    slice_bytes = B.lib.b200shm_heap_slice()
    buf = heap(8)
    with pytest.raises(B.B200Error) as e:
        B.reduce_noalloc("min", "float32", "rec_dbl", 2, B.ptr(0, buf), slice_bytes,
                         B.ptr(0, buf), slice_bytes, LIMIT + 1)
    assert e.value.code == -2 and b"limited to" in B.lib.b200shm_last_error()
