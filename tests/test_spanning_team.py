"""A team spanning GPUs (osss-ucx_b200/spanning.py), its cross-rank steps on
CPU gloo ranks (world sizes 2, 3 and 4).  Each rank's local step -- on a GPU
the engine's reduction over its members -- is stood in for here by the
oracle's restatement over the same members, in the same order; the
butterfly over ranks, the rank-order fold of a world that is not a power of
two, the exactness rule and the write-back run as they do on GPUs.  The
result is compared with the oracle over the whole team: bit for bit where
`exact` says so, else within P * eps * sum|x|."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# (op, dtype, algo, P)
CASES = {
    2: [("sum", "float32", "rec_dbl", 16), ("prod", "float64", "rabenseifner", 8),
        ("sum", "float64", "rabenseifner2", 32), ("xor", "int64", "rec_dbl", 6),
        ("min", "float32", "rec_dbl", 8), ("sum", "float32", "linear", 8),
        ("sum", "float64", "rec_dbl", 12)],
    3: [("sum", "int32", "rec_dbl", 6), ("or", "uint64", "linear", 9),
        ("sum", "float64", "rec_dbl", 6)],
    4: [("sum", "float32", "rec_dbl", 16), ("sum", "float64", "rabenseifner", 64),
        ("prod", "int64", "rec_dbl", 12), ("max", "float64", "linear", 8),
        ("sum", "float32", "rec_dbl", 4)],
}
N = 1000


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def inputs(op, dtype, P, seed):
    import gen
    dt = np.dtype(dtype)
    if dt.kind in "iu":
        lo, hi = (-3, 3) if op == "prod" else (None, None)
        if dt.kind == "u" and lo is not None:
            lo = 0
        return gen.uniform_int(dt, P, N, seed, lo, hi)
    if op == "prod":
        return gen.uniform(dt, P, N, seed, 0.99, 1.01)
    return gen.normal(dt, P, N, seed)


def _rank_main(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    for p in (os.path.join(ROOT, "osss-ucx_b200"), os.path.join(ROOT, "oracle"),
              os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    import oracle
    import spanning
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    rs = oracle.Restatement()

    class OracleLocal(spanning.SpanningTeam):
        """The local step by the oracle (CPU), the write-back into `out`."""

        def local_partial(self, op, dtype, algo, dest, src, nelems):
            return torch.from_numpy(np.ascontiguousarray(rs.reduce(algo, op, self.mine)[0]))

        def write_back(self, result, dest, nelems, dtype):
            self.out = result.numpy().copy()

    res = []
    for k, (op, dtype, algo, P) in enumerate(CASES[world]):
        x = inputs(op, dtype, P, 100 * world + k)
        per = P // world
        team = OracleLocal(None, per)
        team.mine = x[rank * per:(rank + 1) * per]
        exact = team.reduce(op, dtype, algo, 0, 0, N)
        want = rs.reduce(algo, op, x)[0]
        if exact:
            ok = team.out.tobytes() == want.tobytes()
        else:
            w64 = x.astype(np.float64)
            exact_sum = w64.sum(0) if op == "sum" else w64.prod(0) if op == "prod" else want
            bound = P * np.finfo(np.dtype(dtype)).eps * np.abs(w64).sum(0)
            ok = bool((np.abs(team.out.astype(np.float64) - exact_sum) <= bound).all())
        res.append((k, bool(exact), bool(ok)))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, res))


def run_world(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=300) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


def expected_exact(op, dtype, algo, P, world):
    if not dtype.startswith("float") or op in ("min", "max"):
        return True
    pow2 = lambda n: n & (n - 1) == 0
    return algo in ("rec_dbl", "rabenseifner", "rabenseifner2") and pow2(P) and pow2(world)


def check(world):
    out = run_world(world)
    for rank, res in out.items():
        for k, exact, ok in res:
            op, dtype, algo, P = CASES[world][k]
            assert exact == expected_exact(op, dtype, algo, P, world), (world, CASES[world][k])
            assert ok, (world, rank, CASES[world][k])


def test_two_ranks():
    check(2)


def test_three_ranks_fold_in_rank_order():
    check(3)


def test_four_ranks():
    check(4)


@pytest.mark.gpu
def test_engine_steps_on_one_gpu(B, heap, rs):
    """The engine-backed steps on the GPU, in a world of one rank (NCCL):
    the local partial is the engine's reduction over the local members,
    viewed in place as a tensor, and the write-back broadcasts it to every
    local member -- the same bits as b200shm_reduce over those members;
    fcollect and alltoall through the engine's local steps, and atomics
    through the routing, give the oracle's bytes and counts.  The
    peer-memory form (PeerTeam) in the same world: G = 1, the span kernels
    over this GPU's arena alone, barriers through NCCL."""
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "osss-ucx_b200"))
    import spanning
    port = free_port()
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0,
                            world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        for op, dtype, algo, P in (("sum", "float32", "rec_dbl", 8), ("xor", "int64", "linear", 5),
                                   ("max", "float64", "rabenseifner", 16)):
            x = inputs(op, dtype, P, P)
            src, dst = heap(x[0].nbytes), heap(x[0].nbytes)
            team = (10, 3, P)
            B.put_rows(src, x, team=team)
            B.memset(dst, 0x5A, x[0].nbytes, team=team)
            t = spanning.SpanningTeam(B, P, local_start=10, local_stride=3)
            assert t.reduce(op, dtype, algo, dst, src, N)
            got = B.get_rows(dst, x[0].nbytes, x.dtype, team=team)
            want = rs.reduce(algo, op, x)
            assert (got == want[0]).all() and got.tobytes() == np.broadcast_to(
                want[0], want.shape).tobytes(), (op, dtype, algo)
        P, nb = 6, 48
        team = (7, 2, P)
        t = spanning.SpanningTeam(B, P, local_start=7, local_stride=2)
        x = np.random.default_rng(3).integers(0, 256, (P, P * nb), dtype=np.uint8)
        src, dst = heap(P * nb), heap(P * nb)
        B.put_rows(src, x, team=team)
        t.fcollect(dst, src, nb)
        want = rs.fcollect(np.ascontiguousarray(x[:, :nb]))
        assert B.get_rows(dst, P * nb, np.uint8, team=team).tobytes() == want.tobytes()
        t.alltoall(dst, src, nb)
        assert B.get_rows(dst, P * nb, np.uint8, team=team).tobytes() == rs.alltoall(x).tobytes()
        ctr = heap(64 * 8)
        B.memset(ctr, 0, 64 * 8, team=team)
        ops = np.random.default_rng(4).integers(0, [P, 64], (500, 2))
        fetched = t.amo("fetch_add", "int64", ops[:, 0], ctr + ops[:, 1] * 8, np.ones(500))
        hist = np.zeros((P, 64), np.int64)
        np.add.at(hist, (ops[:, 0], ops[:, 1]), 1)
        assert np.array_equal(B.get_rows(ctr, 64 * 8, np.int64, team=team), hist)
        seen = {}
        for (m, c), f in zip(ops.tolist(), fetched.tolist()):
            seen.setdefault((m, c), []).append(f)
        assert all(sorted(v) == list(range(len(v))) for v in seen.values())

        # the peer-memory form in the same world of one: G = 1, its own arena
        # only, barriers through NCCL
        P8, team8 = 8, (7, 2, 8)
        pt = spanning.PeerTeam(B, P8, local_start=7, local_stride=2, scratch_bytes=1 << 14)
        x = inputs("sum", "float32", P8, P8)
        src, dst = heap(x[0].nbytes), heap(x[0].nbytes)
        B.put_rows(src, x, team=team8)
        assert pt.reduce("sum", "float32", "rec_dbl", dst, src, N)
        assert B.get_rows(dst, x[0].nbytes, x.dtype, team=team8).tobytes() == \
            rs.reduce("rec_dbl", "sum", x).tobytes()
        xb = np.random.default_rng(5).integers(0, 256, (P8, P8 * nb), dtype=np.uint8)
        B.put_rows(src, xb, team=team8)
        pt.fcollect(dst, src, nb)
        want = rs.fcollect(np.ascontiguousarray(xb[:, :nb]))
        assert B.get_rows(dst, P8 * nb, np.uint8, team=team8).tobytes() == want.tobytes()
        pt.alltoall(dst, src, nb)
        assert B.get_rows(dst, P8 * nb, np.uint8, team=team8).tobytes() == \
            rs.alltoall(xb).tobytes()
        B.memset(ctr, 0, 64 * 8, team=team)  # members 0..5 of team8 are team's
        fetched = pt.amo("fetch_add", "int64", ops[:, 0], ctr + ops[:, 1] * 8, np.ones(500))
        assert np.array_equal(B.get_rows(ctr, 64 * 8, np.int64, team=team), hist)
        pt.close()
    finally:
        dist.destroy_process_group()


def _movement_rank_main(rank, world, port, q):
    """fcollect, alltoall and routed fetch-adds over a spanning team of
    world x L members; the local steps on a CPU arena per rank."""
    import datetime
    import torch
    import torch.distributed as dist
    for p in (os.path.join(ROOT, "osss-ucx_b200"), os.path.join(ROOT, "oracle"),
              os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    import oracle
    import spanning
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    rs = oracle.Restatement()

    class CpuArena(spanning.SpanningTeam):
        """Each rank's members as rows of a CPU tensor; the local steps by
        plain copies, in the same places the engine writes."""

        def __init__(self, L, slice_bytes, counters):
            super().__init__(None, L)
            self.arena = torch.zeros((L, slice_bytes), dtype=torch.uint8)
            self.ctr = torch.zeros((L, counters), dtype=torch.int64)

        def row(self, i, off, nbytes):
            return self.arena[i, off:off + nbytes]

        def sync_device(self):
            pass

        def local_fcollect(self, dest, src, nbytes):
            L, r = self.local[2], self.rank
            for i in range(L):
                for k in range(L):
                    o = dest + (r * L + k) * nbytes
                    self.arena[i, o:o + nbytes] = self.arena[k, src:src + nbytes]

        def local_alltoall(self, dest, src, nbytes):
            L, r = self.local[2], self.rank
            for j in range(L):
                for k in range(L):
                    d, s = dest + (r * L + k) * nbytes, src + (r * L + j) * nbytes
                    self.arena[j, d:d + nbytes] = self.arena[k, s:s + nbytes]

        def local_amo(self, amo, dtype, pe_local, off, value):
            old = torch.empty(len(pe_local), dtype=torch.int64)
            for n in range(len(pe_local)):  # fetch-add, one at a time
                i, c = int(pe_local[n]), int(off[n]) // 8
                old[n] = self.ctr[i, c]
                self.ctr[i, c] += value[n]
            return old

    res = []
    for L, nb in ((1, 48), (3, 40), (4, 16)):
        P = L * world
        t = CpuArena(L, 1 << 16, 64)
        rng = np.random.default_rng(P * 7 + nb)
        x = rng.integers(0, 256, (P, P * nb), dtype=np.uint8)  # every member's source
        src, dest = 0, 1 << 15
        for i in range(L):
            t.arena[i, src:src + P * nb] = torch.from_numpy(x[rank * L + i])
        t.fcollect(dest, src, nb)
        want = rs.fcollect(np.ascontiguousarray(x[:, :nb]))
        ok_f = all(t.arena[i, dest:dest + P * nb].numpy().tobytes() == want[rank * L + i].tobytes()
                   for i in range(L))
        t.alltoall(dest, src, nb)
        want = rs.alltoall(x)
        ok_a = all(t.arena[i, dest:dest + P * nb].numpy().tobytes() == want[rank * L + i].tobytes()
                   for i in range(L))
        # fetch-adds of 1 from every rank on random (member, counter) targets
        nops = 200
        ops = [np.random.default_rng(1000 * r + P).integers(0, [P, 64], (nops, 2))
               for r in range(world)]
        mine = ops[rank]
        fetched = t.amo("fetch_add", "int64", mine[:, 0], mine[:, 1] * 8, np.ones(nops, np.int64))
        hist = np.zeros((P, 64), np.int64)
        for o in ops:
            np.add.at(hist, (o[:, 0], o[:, 1]), 1)
        ok_c = np.array_equal(t.ctr.numpy(), hist[rank * L:(rank + 1) * L])
        allf = [None] * world
        dist.all_gather_object(allf, (mine.tolist(), fetched.tolist()))
        seen = {}
        for ol, fl in allf:
            for (m, c), f in zip(ol, fl):
                seen.setdefault((m, c), []).append(f)
        ok_p = all(sorted(v) == list(range(len(v))) for v in seen.values())
        res.append((L, nb, ok_f, ok_a, bool(ok_c), ok_p))
    # one rank names a member outside the team: every rank refuses the call
    t = CpuArena(2, 1 << 12, 8)
    bad_pe = np.array([2 * world if rank == 0 else 0])
    try:
        t.amo("fetch_add", "int64", bad_pe, np.zeros(1, np.int64), np.ones(1, np.int64))
        refused = False
    except ValueError:
        refused = True
    res.append((0, 0, refused, refused, refused, refused))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, res))


def run_movement_world(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    ps = [ctx.Process(target=_movement_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=300) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


@pytest.mark.parametrize("world", [2, 3])
def test_spanning_fcollect_alltoall_and_routed_atomics(world):
    """Byte-exact fcollect and alltoall against the oracle over the whole
    team; routed fetch-adds leave every counter at its op count and hand
    out each counter's values exactly once."""
    out = run_movement_world(world)
    for rank, res in out.items():
        for L, nb, ok_f, ok_a, ok_c, ok_p in res:
            assert ok_f and ok_a and ok_c and ok_p, (world, rank, L, nb, ok_f, ok_a, ok_c, ok_p)
