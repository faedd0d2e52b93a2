"""Device barriers and batched atomics through the C ABI."""
import zlib

import numpy as np
import pytest

import gen

pytestmark = pytest.mark.gpu

BARRIERS = ["linear", "complete_tree", "binomial_tree", "knomial_tree", "dissemination"]


@pytest.mark.parametrize("algo", BARRIERS)
def test_barrier_completes_and_is_reusable(B, algo):
    for team in [(0, 1, 1), (0, 1, 2), (0, 1, 3), (0, 1, 8), (5, 3, 17), (0, 1, 64), (0, 1, 256)]:
        for _ in range(3):
            B.barrier(algo, team=team)


def dev_array(B, heap, arr):
    """Place a host array in PE 0's slice and return (offset, device address)."""
    arr = np.ascontiguousarray(arr)
    off = heap(max(arr.nbytes, 16))
    B.put_rows(off, arr.reshape(1, -1).view(np.uint8), team=(0, 1, 1))
    return off, B.ptr(0, off)


def test_fetch_add_counters_and_fetch_permutation(B, heap, rs):
    """Config 3 in miniature: fetch-add on int64 counters at random (PE,
    offset).  Final counters must equal the sequential restatement; per
    counter, the fetched values with increment 1 must be a permutation of
    {c0, ..., c0+k-1}."""
    npes, ncnt, nops = 64, 1024, 1 << 16
    rng = np.random.default_rng(17)
    pe = rng.integers(0, npes, nops).astype(np.int32)
    idx = rng.integers(0, ncnt, nops).astype(np.int64)
    cnt_off = heap(ncnt * 8)
    c0 = rng.integers(-1000, 1000, size=(npes, ncnt)).astype(np.int64)
    B.put_rows(cnt_off, c0, team=(0, 1, npes))
    _, d_pe = dev_array(B, heap, pe)
    _, d_off = dev_array(B, heap, (cnt_off + idx * 8).astype(np.uint64))
    _, d_val = dev_array(B, heap, np.ones(nops, np.int64))
    f_off, d_f = dev_array(B, heap, np.zeros(nops, np.int64))
    B.amo_batch("fetch_add", "int64", nops, d_pe, d_off, d_val, None, d_f)
    final = B.get_rows(cnt_off, ncnt * 8, np.int64, team=(0, 1, npes))
    fetched = B.get_rows(f_off, nops * 8, np.int64, team=(0, 1, 1))[0]
    _, want_final = rs.amo_fetch_add(npes, ncnt, pe, idx, np.ones(nops, np.int64), c0)
    assert np.array_equal(final, want_final)
    key = pe.astype(np.int64) * ncnt + idx
    order = np.lexsort((fetched, key))
    ks, fs = key[order], fetched[order]
    starts = np.r_[0, np.flatnonzero(np.diff(ks)) + 1]
    rank = np.arange(nops) - np.repeat(starts, np.diff(np.r_[starts, nops]))
    assert np.array_equal(fs, c0.reshape(-1)[ks] + rank)


@pytest.mark.parametrize("amo,dt", [("swap", "int64"), ("cswap", "int64"), ("fetch_and", "uint64"),
                                    ("fetch_or", "int32"), ("fetch_xor", "uint32"),
                                    ("fetch", "int64"), ("set", "float64"), ("add", "int32"),
                                    ("inc", "int64"), ("swap", "float32")])
def test_amo_family_on_distinct_targets(B, heap, amo, dt):
    """Each op on distinct words: result and fetched value are determined."""
    npes, nops = 16, 4096
    npdt = {"int64": np.int64, "uint64": np.uint64, "int32": np.int32, "uint32": np.uint32,
            "float64": np.float64, "float32": np.float32}[dt]
    es = np.dtype(npdt).itemsize
    rng = np.random.default_rng(zlib.crc32(f"{amo}{dt}".encode()))
    slots = rng.permutation(npes * nops)[:nops]
    pe = (slots // nops).astype(np.int32)
    idx = (slots % nops).astype(np.int64)
    base = heap(nops * es)
    if np.dtype(npdt).kind == "f":
        init = rng.standard_normal((npes, nops)).astype(npdt)
        val = rng.standard_normal(nops).astype(npdt)
        cond = init[pe, idx]
    else:
        init = gen.uniform_int(npdt, npes, nops, 3)
        val = gen.uniform_int(npdt, 1, nops, 4)[0]
        cond = np.where(rng.random(nops) < 0.5, init[pe, idx], val)
    B.put_rows(base, init, team=(0, 1, npes))
    _, d_pe = dev_array(B, heap, pe)
    _, d_off = dev_array(B, heap, (base + idx * es).astype(np.uint64))
    _, d_val = dev_array(B, heap, val)
    _, d_cond = dev_array(B, heap, cond)
    f_off, d_f = dev_array(B, heap, np.zeros(nops, npdt))
    B.amo_batch(amo, dt, nops, d_pe, d_off, d_val, d_cond, d_f)
    final = B.get_rows(base, nops * es, npdt, team=(0, 1, npes))
    fetched = B.get_rows(f_off, nops * es, npdt, team=(0, 1, 1))[0]
    old = init[pe, idx]
    want = init.copy()
    with np.errstate(over="ignore"):
        if amo in ("swap", "set"):
            want[pe, idx] = val
        elif amo == "cswap":
            want[pe, idx] = np.where(old == cond, val, old)
        elif amo == "fetch_and":
            want[pe, idx] = old & val
        elif amo == "fetch_or":
            want[pe, idx] = old | val
        elif amo == "fetch_xor":
            want[pe, idx] = old ^ val
        elif amo == "add":
            want[pe, idx] = old + val
        elif amo == "inc":
            want[pe, idx] = old + 1
    assert final.tobytes() == want.tobytes()
    if amo.startswith("fetch") or amo in ("swap", "cswap"):
        assert fetched.tobytes() == old.tobytes()


def test_amo_bad_target_is_reported(B, heap):
    _, d_pe = dev_array(B, heap, np.array([10**6], np.int32))
    _, d_off = dev_array(B, heap, np.array([0], np.uint64))
    _, d_val = dev_array(B, heap, np.array([1], np.int64))
    with pytest.raises(B.B200Error):
        B.amo_batch("add", "int64", 1, d_pe, d_off, d_val)


@pytest.mark.parametrize("algo", BARRIERS)
def test_barrier_with_a_member_that_never_arrives_times_out_and_recovers(B, algo):
    """Failure detection without a GPU fault: one member never arrives, every
    wait that depends on it runs out of a 20 ms budget, the call returns
    B200SHM_ERR_TIMEOUT, the flag lines are back at zero, and the same team's
    next barrier completes."""
    old = B.set_wait_budget(0.02)
    try:
        for team, absent in (((0, 1, 8), 5), ((3, 2, 17), 0), ((0, 1, 64), 63)):
            with pytest.raises(B.B200Error) as e:
                B.barrier_absent(algo, absent, team=team)
            assert e.value.code == -6, e.value
            assert B.barrier_flags_nonzero() == 0
            B.barrier(algo, team=team)
            assert B.barrier_flags_nonzero() == 0
    finally:
        B.set_wait_budget(old)
    assert B.set_wait_budget(0) == pytest.approx(old)
