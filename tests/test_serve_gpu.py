"""The serving loop (b200shm_serve_*): every request kind gives what its
per-call entry point gives; a mix of requests in flight together gives, per
request, what the request gives alone; bad requests are refused at enqueue;
the loop exits when idle and comes back on the next request."""
import time

import numpy as np
import pytest

import oracle
from test_reduce_gpu import nan_equal_bytes

pytestmark = pytest.mark.gpu

ES = {"int32": 4, "uint32": 4, "int64": 8, "uint64": 8, "float32": 4, "float64": 8}
NPT = {"int32": np.int32, "uint32": np.uint32, "int64": np.int64, "uint64": np.uint64,
       "float32": np.float32, "float64": np.float64}
SRC_BYTES = 1 << 20
TEAMS = [(4 * k, 1, 4) for k in range(8)] + [(40, 2, 3), (41, 2, 5), (60, 3, 7), (100, 1, 16),
                                             (120, 1, 1)]


@pytest.fixture
def src_region(B, heap):
    """1 MiB of seeded bytes in every PE, with NaNs and signed zeros planted
    in the float views for MIN/MAX."""
    off = heap(SRC_BYTES)
    rng = np.random.default_rng(5)
    x = rng.integers(0, 256, (B.n_pes(), SRC_BYTES), dtype=np.uint8)
    f = x.view(np.float32)
    f[:, ::11] = np.nan
    f[:, 3::13] = -0.0
    f[:, 5::13] = 0.0
    B.put_rows(off, x)
    return off


def random_request(rng, src, dests, heap, max_bytes=16 << 10, kinds=None):
    kind = str(rng.choice(kinds or ["reduce", "fcollect", "alltoall", "put", "get"]))
    team = TEAMS[int(rng.integers(len(TEAMS)))]
    P = team[2]
    if kind == "reduce":
        dt = str(rng.choice(list(ES)))
        op = str(rng.choice(oracle.OPS if dt[0] in "iu" else ["sum", "prod", "min", "max"]))
        algo = str(rng.choice(oracle.ALGOS))
        n = int(rng.integers(1, max_bytes // ES[dt] + 1))
        so = src + int(rng.integers(0, (SRC_BYTES - n * ES[dt]) // ES[dt])) * ES[dt]
        d = heap(n * ES[dt])
        dests.append((d, n * ES[dt], team))
        return dict(kind=kind, op=op, dtype=dt, algo=algo, team=team, src=so, dest=d, n=n)
    if kind in ("fcollect", "alltoall"):
        n = int(rng.integers(1, max_bytes // P + 1))
        sb = n if kind == "fcollect" else P * n
        so = src + int(rng.integers(0, SRC_BYTES - sb))
        d = heap(P * n)
        dests.append((d, P * n, team))
        return dict(kind=kind, team=team, src=so, dest=d, n=n)
    n = int(rng.integers(1, max_bytes + 1))
    a, b = (int(v) for v in rng.integers(0, 128, 2))
    so = src + int(rng.integers(0, SRC_BYTES - n))
    d = heap(n)
    target = b if kind == "put" else a
    dests.append((d, n, (target, 1, 1)))
    return dict(kind=kind, team=(a, 1, 1), pe=b, src=so, dest=d, n=n)


def read_dests(B, dests):
    return [B.get_rows(d, nb, np.uint8, team=team).tobytes() for d, nb, team in dests]


def clear_dests(B, dests):
    for d, nb, team in dests:
        B.memset(d, 0xA5, nb, team=team)


def test_each_kind_matches_per_call(B, heap, src_region):
    rng = np.random.default_rng(1)
    dests, items = [], []
    for kind in ["reduce"] * 24 + ["fcollect", "alltoall", "put", "get"] * 3:
        items.append(random_request(rng, src_region, dests, heap, kinds=[kind]))
    reqs = B.make_requests(items)
    srv = B.Server(queue_slots=64)
    try:
        for k in range(len(items)):
            srv.wait(srv.enqueue(reqs[k]))
    finally:
        srv.stop()
    got = read_dests(B, dests)
    clear_dests(B, dests)
    B.replay(reqs, np.zeros(len(items)))  # per call, one blocking entry point each
    want = read_dests(B, dests)
    for k, (g, w) in enumerate(zip(got, want)):
        assert g == w, (k, items[k])


def test_reduce_matches_oracle(B, heap, rs):
    """Served reductions against the oracle directly (not only through the
    per-call path), float trees and MIN/MAX with NaN included."""
    rng = np.random.default_rng(2)
    srv = B.Server(queue_slots=16)
    try:
        for k, (dt, op, algo, P) in enumerate([("float32", "sum", "rec_dbl", 7),
                                                ("float64", "prod", "binomial", 6),
                                                ("float32", "max", "rec_dbl", 5),
                                                ("float64", "min", "rabenseifner", 12),
                                                ("float32", "sum", "linear", 9),
                                                ("int64", "xor", "rec_dbl", 16),
                                                ("uint32", "prod", "binomial", 3)]):
            N = 3000
            x = rng.standard_normal((P, N)).astype(NPT[dt]) if dt[0] == "f" else \
                rng.integers(0, 1 << 30, (P, N)).astype(NPT[dt])
            if op in ("min", "max"):
                x.reshape(-1)[::17] = np.nan
                x.reshape(-1)[1::19] = -0.0
                x.reshape(-1)[2::19] = 0.0
            if op == "prod" and dt[0] == "f":
                x = (1 + 0.01 * x).astype(x.dtype)
            team = (10 + k, 1, P)
            s, d = heap(x[0].nbytes), heap(x[0].nbytes)
            B.put_rows(s, x, team=team)
            req = B.make_requests([dict(kind="reduce", op=op, dtype=dt, algo=algo, team=team,
                                        src=s, dest=d, n=N)])
            srv.wait(srv.enqueue(req[0]))
            got = B.get_rows(d, x[0].nbytes, x.dtype, team=team)
            want = rs.reduce(algo, op, x)
            assert nan_equal_bytes(got, want), (dt, op, algo, P)
    finally:
        srv.stop()


def test_mix_in_flight_equals_alone(B, heap, src_region):
    """300 requests of every kind, all arriving at once (as many in flight as
    the 128 slots hold), then each replayed alone through the per-call path:
    the bytes of every dest agree; int64 fetch-adds on shared counters add up
    and hand out each counter's values exactly once."""
    rng = np.random.default_rng(3)
    dests, items = [], []
    for _ in range(260):
        items.append(random_request(rng, src_region, dests, heap))
    NC = 16
    ctr = heap(NC * 8)
    B.memset(ctr, 0, NC * 8, team=(0, 1, 8))
    amo_items = [dict(kind="amo", op="fetch_add", dtype="int64", pe=int(rng.integers(8)),
                      dest=ctr + 8 * int(rng.integers(NC)), value=1) for _ in range(40)]
    order = rng.permutation(len(items) + len(amo_items))
    allitems = [(items + amo_items)[i] for i in order]
    reqs = B.make_requests(allitems)
    srv = B.Server(queue_slots=128)
    try:
        lat, fetched = srv.replay(reqs, np.zeros(len(allitems)))
    finally:
        srv.stop()
    assert (lat >= 0).all()
    got = read_dests(B, dests)
    counters = B.get_rows(ctr, NC * 8, np.int64, team=(0, 1, 8))
    seen = {}
    for it, f in zip(allitems, fetched):
        if it["kind"] == "amo":
            seen.setdefault((it["pe"], it["dest"]), []).append(int(f))
    for (pe, off), vals in seen.items():
        assert sorted(vals) == list(range(len(vals)))
        assert counters[pe, (off - ctr) // 8] == len(vals)
    assert counters.sum() == len(amo_items)
    clear_dests(B, dests)
    solo = B.make_requests(items)
    B.replay(solo, np.zeros(len(items)))
    want = read_dests(B, dests)
    for k, (g, w) in enumerate(zip(got, want)):
        assert g == w, (k, items[k])


def test_bad_requests_are_refused(B, heap):
    a = heap(4096)
    srv = B.Server(queue_slots=4)
    try:
        bad = [dict(kind="reduce", op="sum", dtype="int32", team=(250, 1, 8), src=a, dest=a + 1024,
                    n=16),
               dict(kind="reduce", op="xor", dtype="float32", team=(0, 1, 4), src=a,
                    dest=a + 1024, n=16),
               dict(kind="reduce", op="sum", dtype="int32", team=(0, 1, 4), src=a, dest=a + 8,
                    n=16),
               dict(kind="put", team=(0, 1, 1), pe=9999, src=a, dest=a + 1024, n=16),
               dict(kind="amo", op="fetch_add", dtype="int64", pe=0, dest=a + 4, value=1),
               dict(kind="amo", op="fetch_add", dtype="float64", pe=0, dest=a, value=1)]
        for it in bad:
            with pytest.raises(B.B200Error):
                srv.enqueue(B.make_requests([it])[0])
    finally:
        srv.stop()


def test_idle_exit_and_relaunch(B, heap):
    a = heap(4096)
    B.memset(a, 0, 8, team=(0, 1, 1))
    srv = B.Server(queue_slots=4, idle_seconds=0.05)
    try:
        req = B.make_requests([dict(kind="amo", op="fetch_add", dtype="int64", pe=0, dest=a,
                                    value=7)])[0]
        assert srv.wait(srv.enqueue(req)) == 0
        n0 = B.launch_count()
        time.sleep(0.3)  # every CTA idles out
        assert srv.wait(srv.enqueue(req)) == 7
        assert B.launch_count() > n0  # the loop was launched again
    finally:
        srv.stop()
    assert B.get_rows(a, 8, np.int64, team=(0, 1, 1))[0, 0] == 14


def test_other_calls_do_not_wait_for_a_running_loop(B, heap):
    """Batched reductions (stream-ordered plan memory, event-synchronised
    destroy) and collect (stream-ordered size upload) complete while the
    serving loop's kernel keeps running: nothing waits for the device."""
    x = np.arange(4 * 1024, dtype=np.int32).reshape(4, 1024)
    s, d, d2 = heap(x[0].nbytes), heap(x[0].nbytes), heap(4 * x[0].nbytes)
    B.put_rows(s, x, team=(0, 1, 4))
    items = [dict(op="sum", dtype="int32", algo="rec_dbl", team=(0, 1, 4), dest=d, src=s,
                  nelems=1024)]

    def calls():
        b = B.Batch(B.make_descs(items), B.BATCH_GRAPH)
        b.run()
        b.close()
        B.collect(d2, s, [4096] * 4, team=(0, 1, 4))

    calls()  # load the kernels first (CUDA loads a kernel at its first launch)
    srv = B.Server(queue_slots=4, idle_seconds=5.0)
    try:
        t0 = time.perf_counter()
        calls()
        assert time.perf_counter() - t0 < 2.0
    finally:
        srv.stop()
    assert (B.get_rows(d, x[0].nbytes, np.int32, team=(0, 1, 4)) == x.sum(axis=0)).all()
    assert B.get_rows(d2, 4 * x[0].nbytes, np.uint8, team=(0, 1, 4))[1].tobytes() == x.tobytes()


@pytest.mark.parametrize("batch", ["1", "1024"])
def test_mirror_batch_sizes(B, heap, monkeypatch, batch):
    """The mirror copies one request per poll, or up to 1024 (four passes of
    the CTA per step): 3000 fetch-adds arriving at once on 8 counters add up
    and hand out each counter's values exactly once."""
    monkeypatch.setenv("B200SHM_SERVE_MIRROR_BATCH", batch)
    NC = 8
    ctr = heap(NC * 8)
    B.memset(ctr, 0, NC * 8, team=(0, 1, 4))
    rng = np.random.default_rng(int(batch))
    items = [dict(kind="amo", op="fetch_add", dtype="int64", pe=int(rng.integers(4)),
                  dest=ctr + 8 * int(rng.integers(NC)), value=1) for _ in range(3000)]
    srv = B.Server(queue_slots=1024)
    try:
        _, fetched = srv.replay(B.make_requests(items), np.zeros(len(items)))
    finally:
        srv.stop()
    seen = {}
    for it, f in zip(items, fetched):
        seen.setdefault((it["pe"], it["dest"]), []).append(int(f))
    counters = B.get_rows(ctr, NC * 8, np.int64, team=(0, 1, 4))
    for (pe, off), vals in seen.items():
        assert sorted(vals) == list(range(len(vals)))
        assert counters[pe, (off - ctr) // 8] == len(vals)
    assert counters.sum() == len(items)


def test_admission_by_heap_bytes(B, heap, src_region):
    """A server whose heap budget holds one 64 KiB put admits one request at
    a time: each request is claimed on the device only after the previous
    one completed; every put lands; a request above the budget is refused."""
    nb = 64 << 10
    items = [dict(kind="put", team=(k % 8, 1, 1), pe=(5 * k + 3) % 64, src=src_region + 4096 * k,
                  dest=heap(nb), n=nb) for k in range(24)]
    srv = B.Server(queue_slots=64, heap_budget=nb)
    try:
        srv.replay(B.make_requests(items), np.zeros(len(items)))
        tr = [srv.trace(t) for t in range(len(items))]
        with pytest.raises(B.B200Error):
            srv.enqueue(B.make_requests([dict(items[0], n=2 * nb)])[0])
    finally:
        srv.stop()
    for t in range(1, len(items)):
        assert tr[t][1] >= tr[t - 1][2], t  # claimed after the previous one completed
    for it in items:
        got = B.get_rows(it["dest"], nb, np.uint8, team=(it["pe"], 1, 1))
        want = B.get_rows(it["src"], nb, np.uint8, team=(it["team"][0], 1, 1))
        assert got.tobytes() == want.tobytes()


def test_heap_budget_mix_equals_unbudgeted(B, heap, src_region):
    """The mixed stream through a server with a tight heap budget (1 MiB)
    gives the bytes of the same stream through an unbudgeted one."""
    rng = np.random.default_rng(9)
    dests, items = [], []
    for _ in range(120):
        items.append(random_request(rng, src_region, dests, heap, max_bytes=8 << 10))
    budget = 1 << 20  # each request here writes at most 128 KiB of heap
    out = []
    for hb in (budget, 0):
        clear_dests(B, dests)
        srv = B.Server(queue_slots=64, heap_budget=hb)
        try:
            srv.replay(B.make_requests(items), np.zeros(len(items)))
        finally:
            srv.stop()
        out.append(read_dests(B, dests))
    for k, (g, w) in enumerate(zip(*out)):
        assert g == w, (k, items[k])


def test_stop_drains_a_budgeted_loop(B, heap, src_region):
    """Requests still waiting for heap room when the host stops the loop are
    served before it exits: stop drains."""
    nb = 64 << 10
    items = [dict(kind="put", team=(k % 8, 1, 1), pe=(7 * k + 1) % 64, src=src_region + 8192 * k,
                  dest=heap(nb), n=nb) for k in range(12)]
    srv = B.Server(queue_slots=32, heap_budget=nb)
    for r in B.make_requests(items):
        srv.enqueue(r)
    srv.stop()
    for it in items:
        got = B.get_rows(it["dest"], nb, np.uint8, team=(it["pe"], 1, 1))
        want = B.get_rows(it["src"], nb, np.uint8, team=(it["team"][0], 1, 1))
        assert got.tobytes() == want.tobytes()


def test_wait_on_a_ticket_that_never_completes_times_out(B, heap):
    """The host-side bound: waiting on a ticket that was never issued (so it
    never completes) returns B200SHM_ERR_TIMEOUT after the timeout, and the
    server keeps serving afterwards."""
    a = heap(4096)
    B.memset(a, 0, 8, team=(0, 1, 1))
    srv = B.Server(queue_slots=8, idle_seconds=0.05)
    try:
        req = B.make_requests([dict(kind="amo", op="fetch_add", dtype="int64", pe=0, dest=a,
                                    value=3)])[0]
        t = srv.enqueue(req)
        assert srv.wait(t) == 0
        t0 = time.time()
        with pytest.raises(B.B200Error) as e:
            srv.wait(t + 5, timeout=0.05)
        assert e.value.code == -6 and time.time() - t0 < 5.0
        assert srv.poll(t + 5)[0] is False
        assert srv.wait(srv.enqueue(req)) == 3
    finally:
        srv.stop()
    assert B.get_rows(a, 8, np.int64, team=(0, 1, 1))[0, 0] == 6


def test_stream_ordered_per_call_matches_blocking(B, heap, src_region):
    """b200shm_serve_replay_ordered (every request's per-call entry point
    back to back on one stream) leaves what the blocking per-call replay
    leaves, and hands back AMO old values as a permutation."""
    rng = np.random.default_rng(12)
    dests, items = [], []
    for kind in ["reduce"] * 12 + ["fcollect", "alltoall", "put", "get"] * 3:
        items.append(random_request(rng, src_region, dests, heap, kinds=[kind]))
    ctr = heap(8)
    B.memset(ctr, 0, 8, team=(5, 1, 1))
    items += [dict(kind="amo", op="fetch_add", dtype="int64", pe=5, dest=ctr, value=1)] * 16
    reqs = B.make_requests(items)
    B.replay(reqs, np.zeros(len(items)))
    want = read_dests(B, dests)
    clear_dests(B, dests)
    B.memset(ctr, 0, 8, team=(5, 1, 1))
    sec, fetched = B.replay_ordered(reqs[:])  # a slice: a list of requests
    assert sec > 0
    assert read_dests(B, dests) == want
    assert sorted(fetched[-16:].tolist()) == list(range(16))
