"""Data movement and atomics at the configured sizes (128 members), and the
all-to-all forms on teams of 256 and 2048 members.

The 128-member copies at full size are compared with the reference build in
test_parity_reference_gpu.py; here they are compared with the restatement,
so they also run where oracle/_ref is absent."""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import gen

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_alltoallmem_64k_blocks_128_members(B, heap, rs):
    P, blk = 128, 65536
    team = (0, 1, P)
    x = gen.uniform_int(np.uint8, P, P * blk, 41)
    src, dst = heap(x[0].nbytes), heap(x[0].nbytes)
    B.put_rows(src, x, team=team)
    B.memset(dst, 0x5A, x[0].nbytes, team=team)
    B.alltoall(dst, src, blk, team=team)
    got = B.get_rows(dst, x[0].nbytes, np.uint8, team=team)
    assert got.tobytes() == rs.alltoall(x).tobytes()


def test_alltoalls64_dst2_sst3_4096_128_members(B, heap, rs):
    P, n = 128, 4096
    team = (0, 1, P)
    x = gen.uniform_int(np.int64, P, P * n * 3, 42)
    d0 = gen.uniform_int(np.int64, P, P * n * 2, 43)
    src, dst = heap(x[0].nbytes), heap(d0[0].nbytes)
    B.put_rows(src, x, team=team)
    B.put_rows(dst, d0, team=team)
    B.alltoalls(dst, src, 2, 3, n, 8, team=team)
    got = B.get_rows(dst, d0[0].nbytes, np.int64, team=team)
    assert got.tobytes() == rs.alltoalls(x, d0, 2, 3, n).tobytes()


def test_fcollect64_4096_128_members(B, heap, rs):
    P, n = 128, 4096
    team = (0, 1, P)
    x = gen.uniform_int(np.int64, P, n, 44)
    src, dst = heap(x[0].nbytes), heap(x.nbytes)
    B.put_rows(src, x, team=team)
    B.memset(dst, 0x5A, x.nbytes, team=team)
    B.fcollect(dst, src, x[0].nbytes, team=team)
    got = B.get_rows(dst, x.nbytes, np.int64, team=team)
    assert got.tobytes() == rs.fcollect(x).tobytes()


def test_fetch_add_2p20_ops_on_2p20_counters(B, rs):
    """2^20 int64 fetch-adds of 1 at uniformly random (PE, offset) over 2^20
    counters per PE on 128 PEs.  Final counters equal the restatement's
    sequential application; per counter, the fetched values are a
    permutation of {c0, ..., c0 + k - 1}."""
    npes, ncnt, nops = 128, 1 << 20, 1 << 20
    rng = np.random.default_rng(45)
    pe = rng.integers(0, npes, nops).astype(np.int32)
    idx = rng.integers(0, ncnt, nops).astype(np.int64)
    c0 = rng.integers(-1000, 1000, size=(npes, ncnt)).astype(np.int64)
    region = B.malloc(ncnt * 8)  # counters in PEs 0..127; op arrays in PEs 128..131
    try:
        B.put_rows(region, c0, team=(0, 1, npes))
        arrays = [(pe.view(np.uint8), 128), ((region + idx * 8).astype(np.uint64).view(np.uint8), 129),
                  (np.ones(nops, np.int64).view(np.uint8), 130),
                  (np.zeros(nops, np.int64).view(np.uint8), 131)]
        for a, p in arrays:
            B.put_rows(region, a.reshape(1, -1), team=(p, 1, 1))
        B.amo_batch("fetch_add", "int64", nops, B.ptr(128, region), B.ptr(129, region),
                    B.ptr(130, region), None, B.ptr(131, region))
        final = B.get_rows(region, ncnt * 8, np.int64, team=(0, 1, npes))
        fetched = B.get_rows(region, nops * 8, np.int64, team=(131, 1, 1))[0]
    finally:
        B.free(region)
    _, want = rs.amo_fetch_add(npes, ncnt, pe, idx, np.ones(nops, np.int64), c0)
    assert np.array_equal(final, want)
    key = pe.astype(np.int64) * ncnt + idx
    order = np.lexsort((fetched, key))
    ks, fs = key[order], fetched[order]
    starts = np.r_[0, np.flatnonzero(np.diff(ks)) + 1]
    rank = np.arange(nops) - np.repeat(starts, np.diff(np.r_[starts, nops]))
    assert np.array_equal(fs, c0.reshape(-1)[ks] + rank)


@pytest.mark.parametrize("blk,dt", [(1024, np.uint8), (48, np.uint8), (40, np.uint32),
                                    (16, np.int64)])
def test_alltoall_256_members(B, heap, rs, blk, dt):
    """256 members: 65536 pairs, more than one launch grid dimension holds;
    blocks of 1 KiB take the per-pair kernel, small ones the flat kernel."""
    P = 256
    team = (0, 1, P)
    x = gen.uniform_int(dt, P, P * blk // np.dtype(dt).itemsize, blk)
    src, dst = heap(x[0].nbytes), heap(x[0].nbytes)
    B.put_rows(src, x, team=team)
    B.memset(dst, 0x5A, x[0].nbytes, team=team)
    B.alltoall(dst, src, blk, team=team)
    got = B.get_rows(dst, x[0].nbytes, dt, team=team)
    assert got.tobytes() == rs.alltoall(x).tobytes()


@pytest.mark.parametrize("n,dst_s,sst_s,dt", [(5, 2, 3, np.int64), (100, 2, 3, np.int64),
                                              (7, 1, 2, np.int32), (70, 3, 1, np.uint8)])
def test_alltoalls_256_members(B, heap, rs, n, dst_s, sst_s, dt):
    P = 256
    team = (0, 1, P)
    x = gen.uniform_int(dt, P, P * n * sst_s, n)
    d0 = gen.uniform_int(dt, P, P * n * dst_s, n + 1)
    src, dst = heap(x[0].nbytes), heap(d0[0].nbytes)
    B.put_rows(src, x, team=team)
    B.put_rows(dst, d0, team=team)
    B.alltoalls(dst, src, dst_s, sst_s, n, np.dtype(dt).itemsize, team=team)
    got = B.get_rows(dst, d0[0].nbytes, dt, team=team)
    assert got.tobytes() == rs.alltoalls(x, d0, dst_s, sst_s, n).tobytes()


WORLD_2048 = textwrap.dedent("""
    import sys
    import numpy as np
    sys.path[:0] = [{pkg!r}, {orc!r}, {tst!r}]
    import b200shm as B, gen, oracle
    rs = oracle.Restatement()
    P = 2048
    B.init(P, 2 << 20)
    team = (0, 1, P)
    for blk, dt in ((16, np.uint8), (24, np.uint8), (64, np.int64)):
        x = gen.uniform_int(dt, P, P * blk // np.dtype(dt).itemsize, blk)
        src, dst = B.malloc(x[0].nbytes), B.malloc(x[0].nbytes)
        B.put_rows(src, x, team=team)
        B.alltoall(dst, src, blk, team=team)
        got = B.get_rows(dst, x[0].nbytes, dt, team=team)
        assert got.tobytes() == rs.alltoall(x).tobytes(), ("alltoall", blk)
        B.free(src); B.free(dst)
    n = 2
    x = gen.uniform_int(np.int64, P, P * n * 3, 7)
    d0 = gen.uniform_int(np.int64, P, P * n * 2, 8)
    src, dst = B.malloc(x[0].nbytes), B.malloc(d0[0].nbytes)
    B.put_rows(src, x, team=team)
    B.put_rows(dst, d0, team=team)
    B.alltoalls(dst, src, 2, 3, n, 8, team=team)
    got = B.get_rows(dst, d0[0].nbytes, np.int64, team=team)
    assert got.tobytes() == rs.alltoalls(x, d0, 2, 3, n).tobytes(), "alltoalls"
    # barriers over more members than one CTA holds: the cooperative form
    for algo in B.BARRIER_ALGOS:
        for tm in ((0, 1, 2048), (5, 3, 300), (0, 1, 257)):
            for _ in range(2):
                B.barrier(algo, team=tm)
    B.finalize()
    print("ok")
""")


def test_alltoall_2048_member_world():
    """The 2048-PE world of the batching configuration: shmem_alltoallmem /
    alltoalls64 on every PE at once (4M pairs), and barriers over 257-2048
    members (several CTAs, a cooperative launch), in a process of its own."""
    import __graft_entry__
    __graft_entry__.build_library()
    code = WORLD_2048.format(pkg=os.path.join(ROOT, "osss-ucx_b200"),
                             orc=os.path.join(ROOT, "oracle"), tst=os.path.join(ROOT, "tests"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr


BULK_FCOLLECT = textwrap.dedent("""
    import sys
    import numpy as np
    sys.path[:0] = [{pkg!r}, {orc!r}, {tst!r}]
    import b200shm as B, gen, oracle
    rs = oracle.Restatement()
    B.init(256, 8 << 20)
    for P, nb in ((1, 16), (2, 48), (8, 8192), (8, 8208), (13, 40960), (128, 32768),
                  (256, 4096), (64, 100000 // 16 * 16)):
        x = gen.uniform_int(np.uint8, P, nb, P * 31 + nb)
        team = (0, 1, P)
        src, dst = B.malloc(nb), B.malloc(P * nb)
        B.put_rows(src, x, team=team)
        B.memset(dst, 0x5A, P * nb, team=team)
        B.fcollect(dst, src, nb, team=team)
        got = B.get_rows(dst, P * nb, np.uint8, team=team)
        assert got.tobytes() == rs.fcollect(x).tobytes(), (P, nb)
        B.free(src); B.free(dst)
    B.finalize()
    print("ok")
""")


def test_fcollect_staged_through_shared_memory():
    """The fcollect form that stages tiles in shared memory with bulk copies
    (selected by B200SHM_FCOLLECT_BULK=1): single and multiple tiles, a
    partial last tile, 1 to 256 members; bit-exact with the oracle."""
    import __graft_entry__
    __graft_entry__.build_library()
    code = BULK_FCOLLECT.format(pkg=os.path.join(ROOT, "osss-ucx_b200"),
                                orc=os.path.join(ROOT, "oracle"), tst=os.path.join(ROOT, "tests"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, B200SHM_FCOLLECT_BULK="1"))
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
