"""spanning.PeerTeam's host logic on CPU gloo ranks (world sizes 2 and 4):
the exchange of arena handles and scratch offsets, the refusal of ranks
that disagree, the partial addresses, the chunking of long vectors through
the scratch object, and the barrier-separated phases.

Each rank's engine is stood in for by `ShmEngine`: its arena is a POSIX
shared-memory block (so the other ranks can map it, as they map a GPU
arena through CUDA IPC), addresses are (rank + 1) << 40 plus the offset,
its local reduction is the oracle's restatement over its members, and its
span steps restate the span kernels on the mapped arenas -- the combine
with the kernel's relative slots (slot y holds rank y ^ rank's partial;
level l updates the slots whose low l+1 bits are zero).  Results are
compared with the oracle over the whole team, bit for bit where `exact`
says so."""
import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = [("sum", "float32", "rec_dbl", 5000), ("prod", "float64", "rabenseifner", 301),
         ("xor", "int64", "linear", 700), ("min", "int32", "rec_dbl", 999),
         ("max", "float32", "binomial", 64), ("sum", "uint64", "rabenseifner2", 1500),
         ("sum", "int8", "rec_dbl", 3000), ("sum", "float32", "linear", 800)]
L = 4
LOCAL = (1, 2, L)
NPES, SLICE = 8, 1 << 18
TAG = 40


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _np_op(op):
    return {"sum": np.add, "prod": np.multiply, "min": np.minimum, "max": np.maximum,
            "and": np.bitwise_and, "or": np.bitwise_or, "xor": np.bitwise_xor}[op]


class ShmEngine:
    """The engine calls PeerTeam makes, over a shared-memory arena."""

    def __init__(self, name, rank, rs):
        from multiprocessing import shared_memory
        self.shm_mod = shared_memory
        self.rank, self.rs = rank, rs
        self.shm = shared_memory.SharedMemory(name=name, create=True, size=NPES * SLICE)
        self.arenas = {rank: np.ndarray(NPES * SLICE, np.uint8, buffer=self.shm.buf)}
        self.opened = {}
        self.top = 0
        self.calls = []

    # -- arena and handles ---------------------------------------------------
    def heap_slice(self):
        return SLICE

    def n_pes(self):
        return NPES

    def heap_base(self):
        return (self.rank + 1) << TAG

    def ipc_handle(self):
        return self.shm.name.encode()

    def peer_open(self, handle):
        name = bytes(handle).decode()
        r = int(name.rsplit("_", 1)[1])
        m = self.shm_mod.SharedMemory(name=name)
        self.opened[r] = m
        self.arenas[r] = np.ndarray(NPES * SLICE, np.uint8, buffer=m.buf)
        return (r + 1) << TAG

    def peer_close(self, base):
        r = (base >> TAG) - 1
        del self.arenas[r]
        self.opened.pop(r).close()

    def malloc(self, nbytes, align=256):
        off = self.top
        self.top += (nbytes + align - 1) // align * align
        assert self.top <= SLICE
        return off

    def free(self, off):
        pass

    def close(self):
        for m in self.opened.values():
            m.close()
        self.arenas.clear()
        self.shm.close()
        self.shm.unlink()

    # -- memory views ----------------------------------------------------------
    def rows(self, off, nbytes, dtype, team=LOCAL, arena=None):
        a = self.arenas[self.rank if arena is None else arena]
        start, stride, size = team
        return [a[(start + i * stride) * SLICE + off:(start + i * stride) * SLICE + off + nbytes]
                .view(dtype) for i in range(size)]

    def at(self, addr, nbytes):
        r, o = (addr >> TAG) - 1, addr & ((1 << TAG) - 1)
        return self.arenas[r][o:o + nbytes]

    # -- the steps ---------------------------------------------------------------
    def reduce(self, op, dtype, algo, dest, src, n, team):
        self.calls.append("reduce")
        dt = np.dtype(dtype)
        x = np.stack(self.rows(src, n * dt.itemsize, dt, team))
        out = self.rs.reduce(algo, op, x)
        for row, v in zip(self.rows(dest, n * dt.itemsize, dt, team), out):
            row[:] = v

    def span_combine(self, op, dtype, G, rank, partials, dest, n, team):
        self.calls.append("combine")
        dt = np.dtype(dtype)
        w = [self.at(partials[y ^ rank], n * dt.itemsize).view(dt).copy() for y in range(G)]
        lvl = 0
        while (1 << lvl) < G:
            b = 1 << lvl
            for y in range(0, G, 2 * b):
                w[y] = _np_op(op)(w[y], w[y + b])
            lvl += 1
        for row in self.rows(dest, n * dt.itemsize, dt, team):
            row[:] = w[0]

    def span_fcollect(self, G, rank, bases, dest, src, nb, team):
        self.calls.append("fcollect")
        start, stride, size = team
        for m in range(G * size):
            q, k = divmod(m, size)
            blk = self.at(bases[q] + (start + k * stride) * SLICE + src, nb).copy()
            for row in self.rows(dest + m * nb, nb, np.uint8, team):
                row[:] = blk

    def span_alltoall(self, G, rank, bases, dest, src, nb, team):
        self.calls.append("alltoall")
        start, stride, size = team
        drows = self.rows(dest, G * size * nb, np.uint8, team)
        for m in range(G * size):
            q, k = divmod(m, size)
            for j in range(size):
                o = bases[q] + (start + k * stride) * SLICE + src + (rank * size + j) * nb
                drows[j][m * nb:(m + 1) * nb] = self.at(o, nb)


def _rank_main(rank, world, port, tag, q):
    import datetime
    import torch.distributed as dist
    for p in (os.path.join(ROOT, "osss-ucx_b200"), os.path.join(ROOT, "oracle"),
              os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    import oracle
    import spanning
    from test_peer_team_gpu import inputs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    rs = oracle.Restatement()
    eng = ShmEngine("b200peer%s_%d" % (tag, rank), rank, rs)

    class Team(spanning.PeerTeam):
        def sync_device(self):
            pass

    res = []
    try:
        try:
            Team(eng, L, local_start=1, local_stride=1 + (rank == world - 1), scratch_bytes=4096)
            res.append(("mismatch", -1, False, ""))
        except ValueError:
            res.append(("mismatch", -1, True, ""))
        t = Team(eng, L, local_start=LOCAL[0], local_stride=LOCAL[1], scratch_bytes=4096)
        assert t.bases[rank] == eng.heap_base() and len(t.bases) == world
        P = world * L
        mine = slice(rank * L, (rank + 1) * L)
        for k, (op, dtype, algo, n) in enumerate(CASES):
            x = inputs(op, dtype, P, n, 77 * world + k)
            nb = x[0].nbytes
            src, dst = eng.malloc(nb), eng.malloc(nb)
            for row, v in zip(eng.rows(src, nb, x.dtype), x[mine]):
                row[:] = v
            eng.calls.clear()
            exact = t.reduce(op, dtype, algo, dst, src, n)
            chunks = -(-nb // 4096)
            phases = eng.calls == ["reduce", "combine"] * chunks
            got = np.stack(eng.rows(dst, nb, x.dtype))
            want = rs.reduce(algo, op, x)[mine]
            if exact:
                ok = got.tobytes() == want.tobytes()
            else:
                w = x.astype(np.float64)
                bound = P * np.finfo(x.dtype).eps * np.abs(w).sum(0)
                ok = bool((np.abs(got.astype(np.float64) - w.sum(0)) <= bound).all())
            res.append(("reduce", k, bool(ok and phases), (bool(exact), chunks)))
        rng = np.random.default_rng(world)
        for nb in (16, 5):
            x = rng.integers(0, 256, (P, P * nb), dtype=np.uint8)
            src, dst = eng.malloc(P * nb), eng.malloc(P * nb)
            for row, v in zip(eng.rows(src, P * nb, np.uint8), x[mine]):
                row[:] = v
            t.fcollect(dst, src, nb)
            want = rs.fcollect(np.ascontiguousarray(x[:, :nb]))[mine]
            got = np.stack(eng.rows(dst, P * nb, np.uint8))
            res.append(("fcollect", nb, got.tobytes() == want.tobytes(), ""))
            t.alltoall(dst, src, nb)
            got = np.stack(eng.rows(dst, P * nb, np.uint8))
            res.append(("alltoall", nb, got.tobytes() == rs.alltoall(x)[mine].tobytes(), ""))
        t.close()
        res.append(("closed", -1, eng.arenas.keys() == {rank}, ""))
    except Exception as e:
        import traceback
        res.append(("error", -1, False, traceback.format_exc()[-600:]))
    dist.barrier()
    eng.close()
    dist.destroy_process_group()
    q.put((rank, res))


def run_world(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    tag = "%d_%d" % (os.getpid(), port)
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, tag, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=300) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    return out


def check(world):
    out = run_world(world)
    assert sorted(out) == list(range(world))
    for rank, res in out.items():
        assert res[-1][0] != "error", (world, rank, res[-1])
        for kind, k, ok, detail in res:
            assert ok, (world, rank, kind, k, detail)
        for kind, k, ok, (exact, chunks) in (r for r in res if r[0] == "reduce"):
            op, dtype, algo, _ = CASES[k]
            assert exact == (not dtype.startswith("float") or op in ("min", "max")
                             or algo != "linear"), CASES[k]


def test_peer_team_host_logic_two_ranks():
    check(2)


def test_peer_team_host_logic_four_ranks():
    check(4)


def _odd_world_main(rank, world, port, tag, q):
    import datetime
    import torch.distributed as dist
    for p in (os.path.join(ROOT, "osss-ucx_b200"), os.path.join(ROOT, "oracle"),
              os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    import oracle
    import spanning
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    eng = ShmEngine("b200peer%s_%d" % (tag, rank), rank, oracle.Restatement())
    try:
        spanning.PeerTeam(eng, L, local_start=LOCAL[0], local_stride=LOCAL[1],
                          scratch_bytes=4096)
        out = "accepted"
    except ValueError:
        out = "refused"
    dist.barrier()
    eng.close()
    dist.destroy_process_group()
    q.put((rank, out))


def test_peer_team_refuses_a_world_that_is_not_a_power_of_two():
    """Three ranks: the butterfly over GPUs needs a power of two, and every
    rank refuses alike (before any mapping is made)."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    tag = "%d_%d" % (os.getpid(), port)
    ps = [ctx.Process(target=_odd_world_main, args=(r, 3, port, tag, q)) for r in range(3)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=300) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == {0: "refused", 1: "refused", 2: "refused"}
