"""The symmetric-heap allocator on the device (b200shm_malloc / b200shm_free
over heap_core.cuh), and admission by the heap's real free bytes in the
serving loop: a request whose dest the loop allocates waits while the heap
is full and runs once the caller frees room."""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_malloc_free_sequence(B):
    """Random sizes and alignments: offsets aligned and disjoint, every
    object usable in every PE, free bytes back to where they started."""
    free0 = B.lib.b200shm_heap_free_bytes()
    rng = np.random.default_rng(3)
    live = {}
    for step in range(400):
        if live and rng.random() < 0.45:
            off = list(live)[int(rng.integers(len(live)))]
            B.free(off)
            del live[off]
            continue
        nbytes = int(rng.choice([1, 8, 255, 256, 4097, 65536, int(rng.integers(1, 1 << 20))]))
        align = int(rng.choice([256, 256, 1024, 65536]))
        off = B.malloc(nbytes, align)
        assert off % align == 0
        for o, n in live.items():
            assert off + nbytes <= o or o + n <= off, (off, nbytes, o, n)
        live[off] = nbytes
    x = np.arange(64, dtype=np.int64)
    for off in list(live)[:8]:
        if live[off] >= 512:
            B.put_rows(off, np.stack([x + p for p in range(4)]), team=(250, 1, 4))
            got = B.get_rows(off, 512, np.int64, team=(250, 1, 4))
            assert (got == np.stack([x + p for p in range(4)])).all()
    for off in live:
        B.free(off)
    assert B.lib.b200shm_heap_free_bytes() == free0


def test_exhaustion_and_bad_frees(B):
    slice_bytes = B.lib.b200shm_heap_slice()
    with pytest.raises(B.B200Error) as e:
        B.malloc(slice_bytes + 1)
    assert e.value.code == -3
    free0 = B.lib.b200shm_heap_free_bytes()
    offs = []
    while True:  # 1 MiB objects until the heap says no
        try:
            offs.append(B.malloc(1 << 20))
        except B.B200Error as err:
            assert err.code == -3
            break
    assert B.lib.b200shm_heap_free_bytes() < (1 << 20) + 256 * len(offs) or len(offs) > 0
    with pytest.raises(B.B200Error) as e:
        B.free(offs[0] + 256)  # not the start of an object
    assert e.value.code == -1
    for o in offs:
        B.free(o)
    with pytest.raises(B.B200Error) as e:
        B.free(offs[0])  # freed twice
    assert e.value.code == -1
    assert B.lib.b200shm_heap_free_bytes() == free0


ADMISSION = textwrap.dedent("""
    import sys, time
    import numpy as np
    sys.path[:0] = [{pkg!r}, {orc!r}, {tst!r}]
    import b200shm as B, gen, oracle
    rs = oracle.Restatement()
    S = 1 << 20                       # one member's dest: 4 blocks of 256 KiB
    B.init(8, 8 << 20)                # one free block of 8 MiB per PE
    team = (0, 1, 4)
    x = gen.uniform_int(np.uint8, 4, S, 5)
    src = B.malloc(S)
    B.put_rows(src, x, team=team)
    filler = B.malloc(B.lib.b200shm_heap_free_bytes() - 3 * S)   # room for three dests
    assert B.lib.b200shm_heap_free_bytes() == 3 * S
    srv = B.Server(queue_slots=16, idle_seconds=5.0)
    reqs = B.make_requests([dict(kind="alltoall", team=team, src=src, dest=B.SERVE_ALLOC,
                                 n=S // 4)] * 6)
    t = [srv.enqueue(r) for r in reqs]
    offs = [srv.wait(k, timeout=30) for k in t[:3]]   # three fit and run
    assert len(set(offs)) == 3
    time.sleep(0.2)
    assert [srv.poll(k)[0] for k in t[3:]] == [False] * 3, "admitted without room"
    assert B.lib.b200shm_heap_free_bytes() == 0
    want = rs.alltoall(x)
    for o in offs:
        assert B.get_rows(o, S, np.uint8, team=team).tobytes() == want.tobytes()
    B.free(offs[0])                   # room for one more
    offs.append(srv.wait(t[3], timeout=30))
    time.sleep(0.1)
    assert [srv.poll(k)[0] for k in t[4:]] == [False] * 2
    B.free(offs[1]); B.free(offs[2])  # and the last two
    offs += [srv.wait(k, timeout=30) for k in t[4:]]
    for o in offs[3:]:
        assert B.get_rows(o, S, np.uint8, team=team).tobytes() == want.tobytes()
        B.free(o)
    srv.stop()
    B.free(filler); B.free(src)
    assert B.lib.b200shm_heap_free_bytes() == 8 << 20
    B.finalize()
    print("ok")
""")


def test_serving_admission_bound_by_the_heap():
    """Six alltoall requests on a team of 4, each asking the loop for a
    1 MiB dest, on a heap with room for three: three run, three wait in the
    ring until the caller frees dests, then run; every result equals the
    oracle's.  A process of its own, so the heap starts as one free block."""
    import __graft_entry__
    __graft_entry__.build_library()
    code = ADMISSION.format(pkg=os.path.join(ROOT, "osss-ucx_b200"),
                            orc=os.path.join(ROOT, "oracle"), tst=os.path.join(ROOT, "tests"))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
