"""Batched reductions (b200shm_batch_*): every result of a mixed batch is
bit-identical to the per-call b200shm_reduce of the same descriptor, and
therefore to the oracle; descriptors that depend on each other are refused."""
import numpy as np
import pytest

import gen
import oracle
from test_reduce_gpu import nan_equal_bytes

pytestmark = pytest.mark.gpu

NP_T = {"int32": np.int32, "int64": np.int64, "uint32": np.uint32, "uint64": np.uint64,
        "float32": np.float32, "float64": np.float64, "int16": np.int16, "complex64": np.complex64,
        "float80": np.longdouble}


def make_batch(B, heap, rng, n, npes, sizes=(1, 2, 3, 5, 8, 13, 16, 31, 64),
               lengths=(1, 3, 4, 17, 100, 1000, 4099)):
    items, inputs = [], []
    for k in range(n):
        size = int(rng.choice(sizes))
        stride = int(rng.choice([1, 1, 2, 3]))
        while (size - 1) * stride >= npes:
            stride = 1
        start = int(rng.integers(0, npes - (size - 1) * stride))
        dt = str(rng.choice(["int32", "int64", "uint32", "uint64", "float32", "float64",
                             "int16", "complex64", "float80"]))
        if dt.startswith(("int", "uint")):
            op = str(rng.choice(oracle.OPS))
        elif dt == "complex64":
            op = str(rng.choice(["sum", "prod"]))
        else:
            op = str(rng.choice(["sum", "prod", "min", "max"]))
        algo = str(rng.choice(oracle.ALGOS + ["auto"]))
        N = int(rng.choice(lengths))
        x = gen.random_values(NP_T[dt], size, N, 1000 + k)
        if op == "prod" and dt.startswith("float"):
            x = (1.0 + 0.01 * x).astype(x.dtype)
        if op in ("min", "max") and dt.startswith("float") and k % 3 == 0:
            x.reshape(-1)[::7] = np.nan
            x.reshape(-1)[1::5] = -0.0
        mis = int(rng.choice([0, 0, 0, 8]))
        src = heap(x[0].nbytes + 64) + mis
        dst = heap(x[0].nbytes + 64) + mis
        team = (start, stride, size)
        B.put_rows(src, x, team=team)
        items.append(dict(op=op, dtype=dt, algo=algo, team=team, dest=dst, src=src, nelems=N))
        inputs.append(x)
    return items, inputs


def results(B, items, inputs):
    return [B.get_rows(it["dest"], x[0].nbytes, x.dtype, team=it["team"])
            for it, x in zip(items, inputs)]


def per_call(B, items, inputs):
    for it in items:
        algo = "rec_dbl" if it["algo"] == "auto" else it["algo"]
        B.reduce(it["op"], it["dtype"], algo, it["dest"], it["src"], it["nelems"], team=it["team"])
    want = results(B, items, inputs)
    for it, x in zip(items, inputs):
        B.memset(it["dest"], 0x5A, x[0].nbytes, team=it["team"])
    return want


def check_oracle(rs, items, inputs, got, every=7):
    for k in range(0, len(items), every):
        it, x = items[k], inputs[k]
        if it["dtype"] in ("complex64", "float80") or (it["op"] in ("sum", "prod") and
                                          it["dtype"].startswith("float") and
                                          it["algo"] == "binomial"):
            continue  # the oracle's binomial float order is arrival-dependent
        algo = "rec_dbl" if it["algo"] == "auto" else it["algo"]
        assert nan_equal_bytes(got[k], rs.reduce(algo, it["op"], x)), (k, it)


@pytest.mark.parametrize("flags", [0, 1, 2, 3, 4, 6])
def test_batch_matches_per_call_and_oracle(B, heap, rs, flags):
    rng = np.random.default_rng(42 + flags)
    items, inputs = make_batch(B, heap, rng, 160, B.n_pes())
    want = per_call(B, items, inputs)
    descs = B.make_descs(items)
    b = B.Batch(descs, flags)
    for rep in range(2):
        for it, x in zip(items, inputs):  # tuning ran the batch at create: clear again
            B.memset(it["dest"], 0x5A, x[0].nbytes, team=it["team"])
        b.run()
        got = results(B, items, inputs)
        for k, (g, w) in enumerate(zip(got, want)):
            assert g.tobytes() == w.tobytes(), (rep, k, items[k])
    b.close()
    assert all(d.algo >= 0 for d in descs)  # AUTO rewritten to a concrete order
    assert any(d.lanes > 1 for d in descs)
    assert all(d.lanes == 0 for d, it in zip(descs, items)
               if it["dtype"] in ("int16", "complex64", "float80"))
    check_oracle(rs, items, inputs, got)


def test_batch_large_teams(B, heap, rs):
    """Teams up to the whole 256-PE arena: butterflies over 128/256 leaves,
    binomial trees over non-power-of-two teams (one lane, deep stack)."""
    rng = np.random.default_rng(7)
    items, inputs = make_batch(B, heap, rng, 48, B.n_pes(), sizes=(100, 129, 200, 255, 256),
                               lengths=(5, 300, 2048))
    want = per_call(B, items, inputs)
    B.Batch(B.make_descs(items), B.BATCH_NO_TUNE).run()
    got = results(B, items, inputs)
    for k, (g, w) in enumerate(zip(got, want)):
        assert g.tobytes() == w.tobytes(), (k, items[k])
    check_oracle(rs, items, inputs, got, every=3)


def test_batch_graph_counts_its_launches(B, heap):
    rng = np.random.default_rng(3)
    items, inputs = make_batch(B, heap, rng, 24, B.n_pes())
    b = B.Batch(B.make_descs(items), B.BATCH_GRAPH | B.BATCH_NO_TUNE)
    n0 = B.launch_count()
    b.run()
    n1 = B.launch_count()
    b.run()
    assert n1 - n0 >= 2 and B.launch_count() - n1 == n1 - n0
    b.close()


def test_reduce_batch_one_shot(B, heap):
    rng = np.random.default_rng(11)
    items, inputs = make_batch(B, heap, rng, 20, B.n_pes())
    want = per_call(B, items, inputs)
    descs = B.make_descs(items)
    assert B.lib.b200shm_reduce_batch(descs, len(descs), None) == 0
    for g, w in zip(results(B, items, inputs), want):
        assert g.tobytes() == w.tobytes()


def test_batch_rejects_bad_descriptor(B, heap):
    a = heap(1024)
    items = [dict(op="sum", dtype="int32", algo="rec_dbl", team=(0, 1, 4), dest=a, src=a + 4,
                  nelems=16)]
    with pytest.raises(B.B200Error, match="overlap"):
        B.Batch(B.make_descs(items))
    items[0].update(src=a + 512, team=(250, 1, 8))  # past the last PE
    with pytest.raises(B.B200Error):
        B.Batch(B.make_descs(items))


def test_batch_rejects_dependent_descriptors(B, heap):
    """The reductions of a batch run concurrently: a dest that another
    descriptor reads or writes (in any member) is refused; a shared source
    and an in-place descriptor are accepted."""
    a, b, c = heap(4096), heap(4096), heap(4096)

    def d(dest, src, team=(0, 1, 4), n=64):
        return dict(op="sum", dtype="int32", algo="rec_dbl", team=team, dest=dest, src=src,
                    nelems=n)

    for bad in ([d(b, a), d(c, b)],                                  # b written, then read
                [d(b, a), d(b + 128, c)],                            # dests overlap
                [d(b, a, team=(0, 2, 4)), d(a, c, team=(2, 1, 2))],  # through member 2
                [d(a, a), d(c, a + 64)]):                            # in place, read by another
        with pytest.raises(B.B200Error, match="overlap"):
            B.Batch(B.make_descs(bad))
    ok = [d(b, a), d(c, a), d(a + 1024, a + 1024, n=16),
          d(b, a, team=(4, 1, 4))]  # same offsets, other members
    B.Batch(B.make_descs(ok)).close()


def test_fill_uniform_is_seeded_and_in_range(B, heap):
    off = heap(4096 * 8)
    B.fill_uniform(off, "int64", 4096, 7, -1000, 1000, team=(0, 1, 4))
    a = B.get_rows(off, 4096 * 8, np.int64, team=(0, 1, 4))
    B.fill_uniform(off, "int64", 4096, 7, -1000, 1000, team=(0, 1, 4))
    assert (B.get_rows(off, 4096 * 8, np.int64, team=(0, 1, 4)) == a).all()
    assert a.min() >= -1000 and a.max() <= 1000 and len(np.unique(a)) > 1000
    assert not (a[0] == a[1]).all()  # PEs differ
    B.fill_uniform(off, "float32", 4096, 8, 0.999, 1.001, team=(0, 1, 4))
    f = B.get_rows(off, 4096 * 4, np.float32, team=(0, 1, 4))
    assert f.min() >= np.float32(0.999) and f.max() < np.float32(1.001)


def test_tuned_plan_is_reported_and_exact(B, heap, rs):
    """The autotuner (the default) times plans inside the whole batch; the
    plan it reports per descriptor may differ from the heuristic's, and the
    results are the same bits either way."""
    rng = np.random.default_rng(99)
    items, inputs = make_batch(B, heap, rng, 120, B.n_pes())
    want = per_call(B, items, inputs)
    heur = B.make_descs(items)
    B.Batch(heur, B.BATCH_NO_TUNE).close()
    tuned = B.make_descs(items)
    b = B.Batch(tuned)
    for it, x in zip(items, inputs):
        B.memset(it["dest"], 0x5A, x[0].nbytes, team=it["team"])
    b.run()
    b.close()
    got = results(B, items, inputs)
    for k, (g, w) in enumerate(zip(got, want)):
        assert g.tobytes() == w.tobytes(), (k, items[k])
    assert all((d.lanes == 0) == (h.lanes == 0) for d, h in zip(tuned, heur))
    assert all(d.tile in (0, 256, 1024, 4096) for d in tuned)
