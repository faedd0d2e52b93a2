"""b200shm_reduce_noalloc: the all-reduce for callers that cannot allocate
device memory (their runtime owns every device allocation, or they may not
call cudaMalloc at all).  It takes the caller's device buffers and keeps
its only scratch -- the list of order-dependent float MIN/MAX elements -- in
a static device array, so it must give exactly what b200shm_reduce gives,
call after call, and must refuse sizes that array cannot hold.

This file is collected last on purpose: if it fails, a run that stops at
the first failure has already run every other test."""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

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
def test_noalloc_matches_b200shm_reduce_twice(B, heap, rs, op, dt, algo, P, N, in_place):
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
    if not (op == "sum" and np.isnan(x).any()):
        assert want.tobytes() == rs.reduce(algo, op, x).tobytes()
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


def test_noalloc_rejects_overlapping_rows(B, heap):
    """Dest rows that overlap source rows without being the same rows give
    wrong results in a one-pass kernel, so they are refused."""
    sb = B.lib.b200shm_heap_slice()
    buf = heap(4096)
    base = B.ptr(0, buf)
    for dst, dstride, src, sstride in [
            (base + sb + 4, sb, base, sb),     # shifted onto the next member's source row
            (base, sb, base, 2 * sb),          # same base, different strides
            (base + 64, sb, base, sb)]:        # own row, shifted
        with pytest.raises(B.B200Error) as e:
            B.reduce_noalloc("sum", "int32", "rec_dbl", 4, dst, dstride, src, sstride, 256)
        assert e.value.code == -1
    with pytest.raises(B.B200Error) as e:   # row size overflows
        B.reduce_noalloc("sum", "int64", "rec_dbl", 2, base + 2048, sb, base, sb, 1 << 62)
    assert e.value.code == -1


FRESH = textwrap.dedent("""
    import sys
    import numpy as np
    import torch
    sys.path[:0] = [{pkg!r}, {orc!r}]
    import b200shm as B, oracle
    rs = oracle.Restatement()
    assert not B.initialized()
    P, N = 24, 5000
    rng = np.random.default_rng(11)
    cases = [("sum", "float32", "rec_dbl", rng.standard_normal((P, N)).astype(np.float32)),
             ("min", "float64", "rabenseifner",
              np.where(rng.random((P, N)) < 0.3, -0.0, rng.standard_normal((P, N)))),
             ("xor", "int64", "linear", rng.integers(-2**62, 2**62, (P, N), dtype=np.int64))]
    for op, dt, algo, x in cases:
        x = np.ascontiguousarray(x, dtype={{"float32": np.float32, "float64": np.float64,
                                            "int64": np.int64}}[dt])
        nb = x[0].nbytes
        # caller-owned device buffers, allocated by the caller (here torch),
        # with different pitches for the source and dest rows
        sstride, dstride = nb + 256, 2 * nb + 512
        src = torch.zeros(P * sstride, dtype=torch.uint8, device="cuda")
        dst = torch.zeros(P * dstride, dtype=torch.uint8, device="cuda")
        src.view(P, sstride)[:, :nb] = torch.from_numpy(x.view(np.uint8)).cuda()
        want = rs.reduce(algo, op, x)
        for call in range(2):
            dst.fill_(0xA5)
            torch.cuda.synchronize()
            B.reduce_noalloc(op, dt, algo, P, dst.data_ptr(), dstride, src.data_ptr(), sstride, N)
            got = dst.view(P, dstride)[:, :nb].cpu().numpy().copy().view(x.dtype)
            assert got.tobytes() == want.tobytes(), (op, dt, call)
    assert not B.initialized()
    print("ok")
""")


def test_noalloc_in_a_fresh_process_without_init():
    """The documented use: a process that never calls b200shm_init passes its
    own device buffers (source and dest rows at different pitches); the
    result equals the oracle's, on two calls in a row."""
    import __graft_entry__
    __graft_entry__.build_library()
    code = FRESH.format(pkg=os.path.join(ROOT, "osss-ucx_b200"), orc=os.path.join(ROOT, "oracle"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
