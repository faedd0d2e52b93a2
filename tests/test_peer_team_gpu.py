"""A team spanning GPUs through peer memory (spanning.PeerTeam): its ranks
are processes that map each other's arenas with CUDA IPC, and its
cross-rank steps are the engine's span kernels (b200shm_span_combine,
b200shm_span_fcollect, b200shm_span_alltoall) reading the other ranks'
arenas with plain loads, and its atomics one-sided system-scope atomics on
the owner's arena (b200shm_span_amo).

The ranks run here as 2 and 4 processes on one GPU.  That is sound for
these kernels: none of them waits on another rank's kernel (host barriers
over a gloo group separate every phase), so they need not run at the same
time.  Each rank holds `L` members of a team of world x L; the results on
every rank's members are compared with the oracle over the whole team: bit
for bit where the team's `exact` says so (and it must say so for every
integer case and the butterfly float cases here), else within
P * eps * sum|x|."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.abspath(__file__)) + "/.."

# (op, dtype, algo, nelems); the scratch object is 64 KiB, so the longer
# vectors go through the combine in several chunks
CASES = [("sum", "float32", "rec_dbl", 40000), ("sum", "float64", "rabenseifner", 3001),
         ("prod", "float64", "rec_dbl", 777), ("xor", "int64", "linear", 5000),
         ("min", "int32", "rec_dbl", 4097), ("max", "float32", "binomial", 1000),
         ("sum", "uint64", "rabenseifner2", 2500), ("sum", "int8", "rec_dbl", 20003),
         ("and", "uint16", "linear", 999), ("sum", "complex64", "rec_dbl", 1000),
         ("prod", "complex128", "rec_dbl", 300), ("sum", "float32", "linear", 3000),
         ("max", "uint8", "binomial", 17)]
L = 4                       # members per rank: PEs 1, 3, 5, 7 of each engine
LOCAL = (1, 2, L)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def inputs(op, dtype, P, n, seed):
    import gen
    dt = np.dtype(dtype)
    if dt.kind in "iu":
        lo, hi = (-3, 3) if op == "prod" else (None, None)
        return gen.uniform_int(dt, P, n, seed, lo, hi)
    if dt.kind == "c":
        if op == "prod":
            re = gen.uniform(np.float64, P, n, seed, 0.99, 1.01)
            im = gen.uniform(np.float64, P, n, seed + 1, -0.01, 0.01)
        else:
            re, im = gen.normal(np.float64, P, n, seed), gen.normal(np.float64, P, n, seed + 1)
        return (re + 1j * im).astype(dt)
    if op == "prod":
        return gen.uniform(dt, P, n, seed, 0.99, 1.01)
    return gen.normal(dt, P, n, seed)


def _rank_main(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    for p in (os.path.join(ROOT, "osss-ucx_b200"), os.path.join(ROOT, "oracle"),
              os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    res = []
    try:
        import b200shm as B
        import oracle
        import spanning
        torch.cuda.set_device(0)
        B.init(8, 8 << 20)
        rs = oracle.Restatement()
        P = world * L
        mine = slice(rank * L, (rank + 1) * L)

        # an engine that disagrees about the local team: every rank refuses
        try:
            spanning.PeerTeam(B, L, local_start=1, local_stride=1 + (rank == world - 1))
            res.append(("mismatch", -1, False, "not refused"))
        except ValueError:
            res.append(("mismatch", -1, True, ""))

        t = spanning.PeerTeam(B, L, local_start=LOCAL[0], local_stride=LOCAL[1],
                              scratch_bytes=1 << 16)
        for k, (op, dtype, algo, n) in enumerate(CASES):
            x = inputs(op, dtype, P, n, 1000 * world + k)
            nb = x[0].nbytes
            src, dst = B.malloc(nb), B.malloc(nb)
            B.put_rows(src, x[mine], team=LOCAL)
            B.memset(dst, 0x5A, nb, team=LOCAL)
            before = B.launch_count()
            exact = t.reduce(op, dtype, algo, dst, src, n)
            launched = B.launch_count() - before
            got = B.get_rows(dst, nb, x.dtype, team=LOCAL)
            want = rs.reduce(algo, op, x)[mine]
            if exact:
                ok = got.tobytes() == want.tobytes()
            else:
                w = x.astype(np.complex128 if x.dtype.kind == "c" else np.float64)
                ref = w.sum(0) if op == "sum" else w.prod(0)
                eps = np.finfo(x.real.dtype).eps
                bound = P * eps * np.abs(w).sum(0)
                ok = bool((np.abs(got.astype(w.dtype) - ref) <= bound).all())
            res.append(("reduce", k, bool(ok) and launched >= 2, (bool(exact), launched)))
            B.free(src)
            B.free(dst)

        # a second team over the same engines shares the peer mappings; its
        # reduction into a dest 4 bytes off 16-byte alignment takes the
        # element-wise combine; closing it leaves the first team's mappings
        t2 = spanning.PeerTeam(B, L, local_start=LOCAL[0], local_stride=LOCAL[1],
                               scratch_bytes=1 << 16)
        x = inputs("sum", "float32", P, 5001, 77)
        nb = x[0].nbytes
        src, dst = B.malloc(nb), B.malloc(nb + 16)
        B.put_rows(src, x[mine], team=LOCAL)
        assert t2.reduce("sum", "float32", "rec_dbl", dst + 4, src, 5001)
        got = B.get_rows(dst + 4, nb, np.float32, team=LOCAL)
        want = rs.reduce("rec_dbl", "sum", x)[mine]
        res.append(("reduce_unaligned", 0, got.tobytes() == want.tobytes(), ""))
        t2.close()
        B.free(src)
        B.free(dst)

        rng = np.random.default_rng(7 + world)
        for nb in (48, 4096, 3):
            x = rng.integers(0, 256, (P, P * nb), dtype=np.uint8)
            src, dst = B.malloc(P * nb), B.malloc(P * nb)
            B.put_rows(src, x[mine], team=LOCAL)
            B.memset(dst, 0xA5, P * nb, team=LOCAL)
            t.fcollect(dst, src, nb)
            want = rs.fcollect(np.ascontiguousarray(x[:, :nb]))[mine]
            got = B.get_rows(dst, P * nb, np.uint8, team=LOCAL)
            res.append(("fcollect", nb, got.tobytes() == want.tobytes(), ""))
            B.memset(dst, 0xA5, P * nb, team=LOCAL)
            t.alltoall(dst, src, nb)
            want = rs.alltoall(x)[mine]
            got = B.get_rows(dst, P * nb, np.uint8, team=LOCAL)
            res.append(("alltoall", nb, got.tobytes() == want.tobytes(), ""))
            B.free(src)
            B.free(dst)

        # one-sided atomics: every rank's fetch-adds on words of every member
        NCNT, NOPS = 64, 3000
        ctr, ctr32 = B.malloc(NCNT * 8), B.malloc(NCNT * 4)
        B.memset(ctr, 0, NCNT * 8, team=LOCAL)
        B.memset(ctr32, 0, NCNT * 4, team=LOCAL)
        t.barrier()
        all_ops = [np.random.default_rng(500 + r).integers(0, [P, NCNT], (NOPS, 2))
                   for r in range(world)]
        ops = all_ops[rank]
        fetched = t.amo("fetch_add", "int64", ops[:, 0], ctr + ops[:, 1] * 8, np.ones(NOPS))
        t.amo("add", "int32", ops[:, 0], ctr32 + ops[:, 1] * 4, np.full(NOPS, 3))
        t.barrier()
        hist = np.zeros((P, NCNT), np.int64)
        for o in all_ops:
            np.add.at(hist, (o[:, 0], o[:, 1]), 1)
        ok = np.array_equal(B.get_rows(ctr, NCNT * 8, np.int64, team=LOCAL), hist[mine])
        ok = ok and np.array_equal(B.get_rows(ctr32, NCNT * 4, np.int32, team=LOCAL),
                                   3 * hist[mine])
        fl = [None] * world
        dist.all_gather_object(fl, fetched.tolist())
        seen = {}
        for r in range(world):
            for (m, c), f in zip(all_ops[r].tolist(), fl[r]):
                seen.setdefault((m, c), []).append(f)
        ok = ok and all(sorted(v) == list(range(len(v))) for v in seen.values())
        res.append(("amo", 0, bool(ok), ""))
        try:  # a member outside the team: the caller's own call fails
            t.amo("add", "int64", [P], [ctr], [1])
            res.append(("amo_bad_member", 0, False, "not refused"))
        except B.B200Error:
            res.append(("amo_bad_member", 0, True, ""))
        t.close()
    except Exception as e:  # reported, then the group is left in order
        res.append(("error", -1, False, repr(e)))
    try:
        dist.barrier()
        dist.destroy_process_group()
    finally:
        q.put((rank, res))


def run_world(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=600) for _ in ps)
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 4])
def test_peer_team_matches_oracle(world):
    """reduce (every dtype class, butterfly and other orders, several
    chunks), fcollect and alltoall (16-byte and byte paths) over world x 4
    members, each rank's members checked against the oracle; one-sided
    atomics from every rank on every member: exact counts, and each
    counter's fetched values a permutation of 0..count-1."""
    out = run_world(world)
    assert sorted(out) == list(range(world))
    for rank, res in out.items():
        assert res and res[-1][0] != "error", (world, rank, res[-1])
        for kind, k, ok, detail in res:
            assert ok, (world, rank, kind, k, detail,
                        CASES[k] if kind == "reduce" else None)
        n_red = sum(1 for r in res if r[0] == "reduce")
        assert n_red == len(CASES)
        for kind, k, ok, (exact, _) in (r for r in res if r[0] == "reduce"):
            op, dtype, algo, _n = CASES[k]
            want_exact = (not (dtype.startswith("float") or dtype.startswith("complex"))
                          or op in ("min", "max")
                          or algo in ("rec_dbl", "rabenseifner", "rabenseifner2"))
            assert exact == want_exact, (world, CASES[k])


@pytest.mark.gpu
def test_span_calls_refuse_addresses_outside_any_arena(B, heap):
    """A rank base or partial that lies in neither this process's arena nor
    an open peer mapping is refused with ERR_ARG before anything launches.
    Every call here moves zero bytes, so none of them would launch a kernel
    even if the check let the address through."""
    base, sl, npes = B.heap_base(), B.heap_slice(), B.n_pes()
    end = base + npes * sl
    dst, src = heap(4096), heap(4096)
    team = (0, 1, 4)
    good = [base, base + 4 * sl]
    # accepted: rank bases whose members' slices lie in this arena
    B.span_fcollect(2, 0, good, dst, src, 0, team=team)
    B.span_alltoall(2, 0, good, dst, src, 0, team=team)
    B.span_amo("fetch_add", "int64", 2, good, 0, 0, 0, team=team)
    B.span_combine("sum", "float32", 2, 0, [B.ptr(0, src), B.ptr(4, src)], dst, 0, team=team)
    bad_bases = [
        [base, end],                 # just past the arena
        [base, base + (npes - 2) * sl],  # starts inside, its 4 members' slices run past the end
        [base - 4 * sl, base],       # before the arena
    ]
    for bases in bad_bases:
        for call in (lambda: B.span_fcollect(2, 0, bases, dst, src, 0, team=team),
                     lambda: B.span_alltoall(2, 0, bases, dst, src, 0, team=team),
                     lambda: B.span_amo("fetch_add", "int64", 2, bases, 0, 0, 0, team=team)):
            with pytest.raises(B.B200Error) as e:
                call()
            assert e.value.code == -1 and "peer mapping" in str(e.value)
    for partials in ([B.ptr(0, src), end + 4096], [base - 4096, base]):
        with pytest.raises(B.B200Error) as e:
            B.span_combine("sum", "float32", 2, 0, partials, dst, 0, team=team)
        assert e.value.code == -1 and "peer mapping" in str(e.value)
