"""Parity of the data-movement collectives and of the golden fixtures on the
GPU, through the C ABI."""
import os

import numpy as np
import pytest

import gen

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def run_fcollect(B, heap, x, team=None, misalign=0):
    P = x.shape[0]
    nb = x[0].nbytes
    team = team or (0, 1, P)
    src = heap(nb + 64) + misalign
    dst = heap(nb * P + 64) + misalign
    B.put_rows(src, x, team=team)
    B.memset(dst, 0x5A, nb * P, team=team)
    B.fcollect(dst, src, nb, team=team)
    return B.get_rows(dst, nb * P, x.dtype, team=team)


def run_alltoall(B, heap, x, team=None, misalign=0):
    P = x.shape[0]
    nb = x[0].nbytes
    team = team or (0, 1, P)
    src = heap(nb + 64) + misalign
    dst = heap(nb + 64) + misalign
    B.put_rows(src, x, team=team)
    B.memset(dst, 0x5A, nb, team=team)
    B.alltoall(dst, src, nb // P, team=team)
    return B.get_rows(dst, nb, x.dtype, team=team)


def run_alltoalls(B, heap, x, d0, dst_s, sst_s, n, team=None):
    P = x.shape[0]
    team = team or (0, 1, P)
    src = heap(x[0].nbytes)
    dst = heap(d0[0].nbytes)
    B.put_rows(src, x, team=team)
    B.put_rows(dst, d0, team=team)
    B.alltoalls(dst, src, dst_s, sst_s, n, x.itemsize, team=team)
    return B.get_rows(dst, d0[0].nbytes, d0.dtype, team=team)


def test_golden_fixtures_on_gpu(B, heap):
    z = np.load(os.path.join(GOLDEN, "config1.npz"))
    src = heap(4096)
    dst = heap(4096)
    B.put_rows(src, z["reduce_in"], team=(0, 1, 8))
    B.reduce("sum", "int32", "rec_dbl", dst, src, 1024, team=(0, 1, 8))
    assert B.get_rows(dst, 4096, np.int32, team=(0, 1, 8)).tobytes() == z["reduce_out"].tobytes()
    assert run_fcollect(B, heap, z["fcollect_in"]).tobytes() == z["fcollect_out"].tobytes()
    B.barrier("binomial_tree", team=(0, 1, 8))
    c = np.load(os.path.join(GOLDEN, "copy.npz"))
    assert run_fcollect(B, heap, c["fcollect/in"]).tobytes() == c["fcollect/out"].tobytes()
    assert run_alltoall(B, heap, c["alltoall/in"]).tobytes() == c["alltoall/out"].tobytes()
    got = run_alltoalls(B, heap, c["alltoalls/in"], c["alltoalls/dest0"], 2, 3, 5)
    assert got.tobytes() == c["alltoalls/out"].tobytes()


def test_golden_reduce_fixtures_on_gpu(B, heap):
    from test_reduce_gpu import gpu_reduce, nan_equal_bytes
    z = np.load(os.path.join(GOLDEN, "reduce.npz"))
    names = sorted({k.rsplit("/", 1)[0] for k in z.files})
    for name in names:
        parts = name.split("/")
        algo, op = (parts[1], parts[2]) if parts[0] == "special" else (parts[0], parts[1])
        x, y = z[name + "/in"], z[name + "/out"]
        got = gpu_reduce(B, heap, algo, op, x)
        if parts[0] == "special":
            assert got.tobytes() == y.tobytes(), name
        else:
            assert nan_equal_bytes(got, y), name


@pytest.mark.parametrize("P,nb", [(1, 16), (2, 48), (3, 5), (8, 2048), (13, 100), (128, 4096)])
def test_fcollect(B, heap, rs, P, nb):
    x = gen.uniform_int(np.uint8, P, nb, P * 7 + nb)
    assert run_fcollect(B, heap, x).tobytes() == rs.fcollect(x).tobytes()
    if P <= 64:
        assert run_fcollect(B, heap, x, misalign=3).tobytes() == rs.fcollect(x).tobytes()


def test_fcollect_strided_team(B, heap, rs):
    x = gen.uniform_int(np.int64, 9, 33, 5)
    assert run_fcollect(B, heap, x, team=(4, 3, 9)).tobytes() == rs.fcollect(x).tobytes()


@pytest.mark.parametrize("P,blk", [(1, 16), (2, 32), (3, 7), (6, 24), (16, 4096), (128, 1024)])
def test_alltoall(B, heap, rs, P, blk):
    x = gen.uniform_int(np.uint8, P, P * blk, P + blk)
    assert run_alltoall(B, heap, x).tobytes() == rs.alltoall(x).tobytes()
    assert run_alltoall(B, heap, x, misalign=1).tobytes() == rs.alltoall(x).tobytes()


def test_alltoall_strided_team(B, heap, rs):
    x = gen.uniform_int(np.uint32, 5, 5 * 12, 3)
    assert run_alltoall(B, heap, x, team=(7, 11, 5)).tobytes() == rs.alltoall(x).tobytes()


@pytest.mark.parametrize("P,n,dst,sst,dt", [(1, 3, 1, 1, np.int64), (4, 5, 2, 3, np.int64),
                                            (6, 17, 3, 1, np.int32), (8, 64, 1, 4, np.int16),
                                            (3, 9, 2, 2, np.uint8), (16, 33, 2, 3, np.int64)])
def test_alltoalls(B, heap, rs, P, n, dst, sst, dt):
    x = gen.uniform_int(dt, P, P * n * sst, P * n)
    d0 = gen.uniform_int(dt, P, P * n * dst, P * n + 1)
    got = run_alltoalls(B, heap, x, d0, dst, sst, n)
    assert got.tobytes() == rs.alltoalls(x, d0, dst, sst, n).tobytes()


@pytest.mark.parametrize("P,root,nb", [(1, 0, 16), (5, 2, 100), (8, 7, 4096), (64, 13, 48)])
def test_broadcast(B, heap, rs, P, root, nb):
    x = gen.uniform_int(np.uint8, P, nb, nb)
    d0 = gen.uniform_int(np.uint8, P, nb, nb + 1)
    src = heap(nb)
    dst = heap(nb)
    B.put_rows(src, x, team=(0, 1, P))
    B.put_rows(dst, d0, team=(0, 1, P))
    B.broadcast(root, dst, src, nb, team=(0, 1, P))
    got = B.get_rows(dst, nb, np.uint8, team=(0, 1, P))
    assert got.tobytes() == rs.broadcast(x, d0, root).tobytes()


def test_copy_argument_errors(B, heap):
    a = heap(1024)
    with pytest.raises(B.B200Error):
        B.fcollect(a, a, 64, team=(0, 1, 4))  # overlap
    with pytest.raises(B.B200Error):
        B.alltoalls(a, a + 512, 0, 1, 4, 8, team=(0, 1, 2))  # zero stride
    with pytest.raises(B.B200Error):
        B.broadcast(9, a, a + 512, 64, team=(0, 1, 4))  # root not a member


@pytest.mark.parametrize("team,counts,align", [
    ((0, 1, 4), [16, 32, 0, 48], 16),          # 16-byte words, one member empty
    ((3, 2, 5), [8, 24, 40, 8, 16], 8),        # 8-byte words, strided team
    ((10, 3, 6), [12, 4, 28, 20, 0, 8], 4),    # 4-byte words
    ((0, 1, 7), [3, 1, 5, 7, 2, 9, 4], 1),     # bytes
    ((255, 1, 1), [1000], 8),                  # one member
])
def test_collect_matches_oracle(B, heap, rs, team, counts, align):
    """Variable-size allgather: member k contributes counts[k] bytes; every
    member's dest holds the contributions concatenated in member order."""
    P = team[2]
    rng = np.random.default_rng(sum(counts) + P)
    src_bytes = max(max(counts), 16)
    x = rng.integers(0, 256, (P, src_bytes), dtype=np.uint8)
    total = sum(counts)
    s = heap(src_bytes + 64) + (align if align < 16 else 0)
    d = heap(total + 64) + (align if align < 16 else 0)
    B.put_rows(s, x, team=team)
    B.memset(d, 0x77, total + 16, team=team)
    B.collect(d, s, counts, team=team)
    got = B.get_rows(d, total + 16, np.uint8, team=team)
    want = rs.collect(x, counts, total + 16)
    want[:, total:] = 0x77
    assert got.tobytes() == want.tobytes()


def test_collect_rejects_bad_arguments(B, heap):
    a = heap(4096)
    with pytest.raises(B.B200Error):
        B.collect(a, a + 64, [64, 64, 64], team=(0, 1, 3))  # dest overlaps source
    with pytest.raises(ValueError):
        B.collect(a, a + 2048, [8, 8], team=(0, 1, 3))      # one size per member
