"""b200shm_reduce_host (host rows in, host rows out, chunked and pipelined)
gives the bits of put_host + b200shm_reduce + get_host, across chunk
boundaries included: the order-dependent float MIN/MAX elements of the
Rabenseifner orders depend on an element's position in the whole vector."""
import numpy as np
import pytest

import gen
import oracle
from test_reduce_gpu import nan_equal_bytes

pytestmark = pytest.mark.gpu

CASES = [("float32", "sum", "rec_dbl", 8), ("float64", "max", "rabenseifner", 6),
         ("float32", "min", "rabenseifner2", 5), ("float64", "prod", "binomial", 7),
         ("int64", "xor", "rec_dbl", 16), ("int32", "sum", "linear", 3),
         ("float32", "max", "rec_dbl", 12)]


@pytest.mark.parametrize("dt,op,algo,P", CASES)
def test_reduce_host_matches_three_calls(B, heap, rs, monkeypatch, dt, op, algo, P):
    monkeypatch.setenv("B200SHM_HOST_CHUNK_BYTES", str(64 << 10))  # many chunks
    N = 20011
    x = gen.random_values(oracle.NP[dt], P, N, 31 + P)
    if op in ("min", "max"):
        x.reshape(-1)[::13] = np.nan
        x.reshape(-1)[1::17] = -0.0
        x.reshape(-1)[2::17] = 0.0
    if op == "prod" and dt.startswith("float"):
        x = (1.0 + 0.01 * x).astype(x.dtype)
    team = (9, 2, P)
    s, d = heap(x[0].nbytes), heap(x[0].nbytes)
    got = B.reduce_host(op, dt, algo, d, s, x, team=team)
    # the three-call form on other objects
    s2, d2 = heap(x[0].nbytes), heap(x[0].nbytes)
    B.put_rows(s2, x, team=team)
    B.reduce(op, dt, algo, d2, s2, N, team=team)
    want = B.get_rows(d2, x[0].nbytes, x.dtype, team=team)
    assert got.tobytes() == want.tobytes()
    if not (op in ("sum", "prod") and dt.startswith("float") and algo == "binomial"):
        assert nan_equal_bytes(got, rs.reduce(algo, op, x))
    # the arena objects hold the same as the host rows
    assert B.get_rows(d, x[0].nbytes, x.dtype, team=team).tobytes() == got.tobytes()


def test_reduce_host_in_place_and_stream(B, heap):
    import torch
    x = gen.random_values(np.int64, 4, 5000, 3)
    s = heap(x[0].nbytes)
    stream = torch.cuda.Stream()
    out = B.reduce_host("sum", "int64", "rec_dbl", s, s, x, team=(0, 1, 4),
                        stream=stream.cuda_stream)
    stream.synchronize()
    assert (out == x.sum(axis=0, dtype=np.int64)[None, :]).all()
