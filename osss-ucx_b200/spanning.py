"""A team whose members span GPUs: P members over G ranks (one process per
GPU), P/G contiguous members on each rank, each rank's members being PEs of
its own engine (b200shm.init on its GPU).

The reference runs a team's reduction as log2(P) rounds between PEs
(reduce_helper_*_rec_dbl, src/shcoll/src/reduce.c:182-293: fold the extra
PEs, then a butterfly whose level l pairs the members that differ in bit
l).  With the members partitioned in contiguous blocks of a power of two,
the butterfly's low levels stay inside one GPU and its high levels pair
whole GPUs.  So a spanning reduction is:

  1. on each GPU, the engine's one-pass reduction over the local members
     (b200shm_reduce over the local team): every local member then holds
     the value of its own subtree -- the butterfly's local levels, in the
     algorithm's order;
  2. across GPUs, the butterfly's remaining levels on those partials:
     log2(G) rounds, round j exchanging the partial with rank r ^ 2^j and
     combining op(own, partner), as every member does in the reference;
  3. on each GPU, the result written to every local member's dest.

Bit-exactness (the cases `exact` names): integer ops and the float ops
whose result does not depend on operand order give the reference's bits
for any team; float SUM/PROD in a butterfly order (rec_dbl, rabenseifner,
rabenseifner2 share the tree) give them when P and G are powers of two and
G divides P, because then steps 1-2 build exactly the reference's tree.
Otherwise (float linear/binomial orders, teams that are not a power of
two, float MIN/MAX over NaN or mixed-sign zeros) the result is within
P * eps * sum|x| of the exact sum, the bound of the reference's own
arrival-order binomial reduction.  Ranks that are not a power of two
combine the partials by an all-gather and a left fold in rank order.

The data movement follows the same split: fcollect gathers the local
members' blocks with the engine and all-gathers the local concatenation
across ranks; alltoall moves the blocks between local members with the
engine and the rest in one all-to-all across ranks; atomics are routed to
the rank that owns their target member and run there as one batch, their
old values returned in the caller's order.  All three are byte-exact for
any team.

SpanningTeam's step 2 moves N elements per round through torch.distributed
(NCCL point-to-point over NVLink on GPUs).  PeerTeam does the cross-GPU
steps in the engine instead: the ranks map each other's arenas through CUDA
IPC, and one kernel per rank reads the other ranks' partials (or blocks)
with plain loads and writes its own members -- the butterfly's cross-GPU
levels fused with the write-back.  No TMA multicast is used anywhere on
this path.  The cross-rank logic runs on gloo ranks on the CPU
(tests/test_spanning_team.py, tests/test_peer_team_cpu.py); PeerTeam's
kernels run as 2 and 4 processes sharing one GPU, which is sound because no
kernel waits on another rank's (tests/test_peer_team_gpu.py).
"""
import torch
import torch.distributed as dist

BUTTERFLY = ("rec_dbl", "rabenseifner", "rabenseifner2")


def _pow2(n):
    return n > 0 and n & (n - 1) == 0


def combine(op, own, other):
    """op(own, partner) with the reference's element operators
    (src/shcoll/src/reduce.c:730-736): a<b?a:b for MIN, a>b?a:b for MAX."""
    if op == "sum":
        return own + other
    if op == "prod":
        return own * other
    if op == "min":
        return torch.where(own < other, own, other)
    if op == "max":
        return torch.where(own > other, own, other)
    if op == "and":
        return torch.bitwise_and(own, other)
    if op == "or":
        return torch.bitwise_or(own, other)
    if op == "xor":
        return torch.bitwise_xor(own, other)
    raise ValueError(op)


_WIRE = {torch.uint16: torch.int16, torch.uint32: torch.int32, torch.uint64: torch.int64}


def butterfly_allreduce(t, op, group=None):
    """Combine every rank's tensor `t` (same shape and dtype on all ranks):
    the butterfly over ranks for a power-of-two world, an all-gather and a
    left fold in rank order otherwise.  Returns the combined tensor.
    Unsigned words travel as the signed type of their width (same bits)."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if world == 1:
        return t
    wire = _WIRE.get(t.dtype)
    if wire is not None:
        return _unwire(butterfly_allreduce_wire(t.view(wire), op, group, t.dtype), t.dtype)
    return butterfly_allreduce_wire(t, op, group, t.dtype)


def _unwire(t, dtype):
    return t.view(dtype) if t.dtype != dtype else t


def butterfly_allreduce_wire(t, op, group, dtype):
    """butterfly_allreduce on tensors in their wire type; the combine runs in
    the element type `dtype`."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    if _pow2(world):
        buf = torch.empty_like(t)
        for j in range(world.bit_length() - 1):
            peer = rank ^ (1 << j)
            gpeer = dist.get_global_rank(group, peer) if group is not None else peer
            reqs = dist.batch_isend_irecv([dist.P2POp(dist.isend, t, gpeer, group),
                                           dist.P2POp(dist.irecv, buf, gpeer, group)])
            for r in reqs:
                r.wait()
            t = combine(op, _unwire(t, dtype), _unwire(buf, dtype)).view(t.dtype)
        return t
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    acc = _unwire(parts[0], dtype)
    for p in parts[1:]:
        acc = combine(op, acc, _unwire(p, dtype))
    return acc


class SpanningTeam:
    """P members over the ranks of `group`, `members_per_rank` on each, which
    are the PEs local_start + i*local_stride (i < members_per_rank) of each
    rank's engine."""

    def __init__(self, engine, members_per_rank, group=None, local_start=0, local_stride=1):
        self.B = engine
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.local = (local_start, local_stride, members_per_rank)
        self.size = members_per_rank * self.world

    def exact(self, op, dtype, algo):
        """True when the result is bit-identical to the reference's."""
        if not dtype.startswith("float") and not dtype.startswith("complex"):
            return True
        if op in ("min", "max"):
            return True  # except over NaN or mixed-sign zeros
        return (algo in BUTTERFLY and _pow2(self.size) and _pow2(self.world)
                and self.size % self.world == 0)

    # -- the three steps; the engine-backed forms run on the rank's GPU ------
    def local_partial(self, op, dtype, algo, dest, src, nelems):
        """Step 1: the engine's reduction over the local members; returns
        member 0's dest as a tensor (on the GPU, sharing the arena)."""
        start, stride, size = self.local
        self.B.reduce(op, dtype, algo, dest, src, nelems, team=(start, stride, size))
        return _device_tensor(self.B.ptr(start, dest), nelems, dtype)

    def write_back(self, result, dest, nelems, dtype):
        """Step 3: the result into member 0's dest, then broadcast to the
        other local members."""
        start, stride, size = self.local
        view = _device_tensor(self.B.ptr(start, dest), nelems, dtype)
        view.copy_(result)
        torch.cuda.synchronize()
        es = torch.empty((), dtype=_TORCH[dtype]).element_size()
        self.B.broadcast(0, dest, dest, nelems * es, team=(start, stride, size))

    def reduce(self, op, dtype, algo, dest, src, nelems):
        """All-reduce over the spanning team; returns True when the result is
        bit-identical to the reference's (see `exact`)."""
        partial = self.local_partial(op, dtype, algo, dest, src, nelems)
        result = butterfly_allreduce(partial.clone(), op, self.group)
        self.write_back(result, dest, nelems, dtype)
        return self.exact(op, dtype, algo)

    # -- data movement (byte-exact for any team) -------------------------------
    def row(self, i, off, nbytes):
        """Local member i's `nbytes` at offset `off`, as a uint8 tensor view."""
        start, stride, _ = self.local
        return _device_tensor(self.B.ptr(start + i * stride, off), nbytes, "uint8")

    def local_fcollect(self, dest, src, nbytes):
        """The local members' blocks in their global places of every local
        member's dest: the engine's fcollect over the local team."""
        start, stride, size = self.local
        self.B.fcollect(dest + self.rank * size * nbytes, src, nbytes, team=(start, stride, size))

    def local_alltoall(self, dest, src, nbytes):
        """The blocks between local members: the engine's alltoall over the
        local team on the local part of the block index."""
        start, stride, size = self.local
        o = self.rank * size * nbytes
        self.B.alltoall(dest + o, src + o, nbytes, team=(start, stride, size))

    def sync_device(self):
        torch.cuda.synchronize()

    def fcollect(self, dest, src, nbytes):
        """Every member's dest holds the P members' blocks in member order
        (fcollect_helper_*, src/shcoll/src/fcollect.c:32-484): the local
        members' blocks by the engine, then one all-gather of the local
        concatenation across ranks, written into every local member."""
        L = self.local[2]
        self.local_fcollect(dest, src, nbytes)
        self.sync_device()
        mine = self.row(0, dest + self.rank * L * nbytes, L * nbytes).clone()
        parts = [torch.empty_like(mine) for _ in range(self.world)]
        dist.all_gather(parts, mine, group=self.group)
        for i in range(L):
            d = self.row(i, dest, self.world * L * nbytes)
            for r, part in enumerate(parts):
                if r != self.rank:
                    d[r * L * nbytes:(r + 1) * L * nbytes].copy_(part)
        self.sync_device()

    def alltoall(self, dest, src, nbytes):
        """Member j's dest block k = member k's source block j
        (alltoall_helper_*, src/shcoll/src/alltoall.c:75-201): the blocks
        between local members by the engine, the rest in one all-to-all
        across ranks (rank r sends rank q the L x L blocks its members hold
        for q's members)."""
        L, G, r, B = self.local[2], self.world, self.rank, nbytes
        self.local_alltoall(dest, src, nbytes)
        self.sync_device()
        srows = [self.row(i, src, G * L * B) for i in range(L)]
        # send[q] = [my member k][q's member j] blocks (q == r: unused)
        send = torch.stack([torch.stack([srows[i][q * L * B:(q + 1) * L * B] for i in range(L)])
                            for q in range(G)]).reshape(-1)
        recv = torch.empty_like(send)
        dist.all_to_all_single(recv, send, group=self.group)
        recv = recv.view(G, L, L, B)  # [sender rank q][its member k][my member j]
        drows = [self.row(j, dest, G * L * B) for j in range(L)]
        for q in range(G):
            if q == r:
                continue
            blk = recv[q]
            for j in range(L):
                drows[j][q * L * B:(q + 1) * L * B].copy_(blk[:, j, :].reshape(-1))
        self.sync_device()

    # -- atomics routed to the rank that owns the target ----------------------
    def local_amo(self, amo, dtype, pe_local, off, value):
        """Run a batch of atomics on this rank's members (the engine's
        b200shm_amo_batch, 8-byte operands); returns the old values (int64,
        on the CPU)."""
        start, stride, _ = self.local
        n = len(pe_local)
        if n == 0:
            return torch.zeros(0, dtype=torch.int64)
        pe = (start + pe_local.to(torch.int64) * stride).to(torch.int32).cuda()
        o = off.to(torch.int64).cuda()  # byte offsets, read by the engine as uint64
        v = value.to(torch.int64).cuda()
        # written whole by the engine's stream: no fill kernel on torch's
        f = torch.empty(n, dtype=torch.int64, device="cuda")
        self.B.amo_batch(amo, dtype, n, pe.data_ptr(), o.data_ptr(), v.data_ptr(), None,
                         f.data_ptr())
        return f.cpu()

    def amo(self, amo, dtype, pe, off, value):
        """Atomics on (member, offset) targets anywhere in the team: each op
        goes to the rank that owns its member (member // members_per_rank),
        which runs its share as one batch; the old values come back in the
        caller's order.  Ops on one word from different ranks are applied in
        an unspecified order, as concurrent AMOs from different PEs are in
        OpenSHMEM (src/shmemc/ucx/comms.c:409-671)."""
        L, G = self.local[2], self.world
        # the exchanges run where the group's backend wants its tensors
        dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
        pe = torch.as_tensor(pe, dtype=torch.int64)
        off = torch.as_tensor(off, dtype=torch.int64)
        value = torch.as_tensor(value, dtype=torch.int64)
        # every rank learns whether any rank has a bad target, so all of them
        # refuse together instead of leaving the others in the exchange
        bad = torch.tensor([int(len(pe) > 0 and (int(pe.min()) < 0 or
                                                 int(pe.max()) >= self.size))], device=dev)
        dist.all_reduce(bad, op=dist.ReduceOp.MAX, group=self.group)
        if int(bad.item()):
            raise ValueError("amo: a target member outside the team of %d" % self.size)
        owner = pe // L
        order = torch.argsort(owner, stable=True)
        send_counts = torch.bincount(owner, minlength=G).to(dev)
        recv_counts = torch.empty_like(send_counts)
        dist.all_to_all_single(recv_counts, send_counts, group=self.group)
        sc, rc = send_counts.tolist(), recv_counts.tolist()
        packed = torch.stack([pe[order] % L, off[order], value[order]], dim=1).to(dev)
        incoming = torch.empty((sum(rc), 3), dtype=torch.int64, device=dev)
        dist.all_to_all_single(incoming, packed, output_split_sizes=rc, input_split_sizes=sc,
                               group=self.group)
        incoming = incoming.cpu()
        fetched_here = self.local_amo(amo, dtype, incoming[:, 0], incoming[:, 1],
                                      incoming[:, 2]).to(dev)
        back = torch.empty(len(pe), dtype=torch.int64, device=dev)
        dist.all_to_all_single(back, fetched_here, output_split_sizes=sc, input_split_sizes=rc,
                               group=self.group)
        out = torch.empty(len(pe), dtype=torch.int64)
        out[order] = back.cpu()
        return out


class PeerTeam(SpanningTeam):
    """The spanning team with its cross-GPU steps as kernels of the engine
    that read the other ranks' arenas directly, through CUDA IPC mappings
    (b200shm_ipc_handle / b200shm_peer_open): plain loads over NVLink, no
    multicast, and no copy through a collective library.

    Every rank's engine has the same npes and heap size and is not in
    managed memory; G = the group's size is a power of two up to 16.  The
    host keeps the phases apart with a barrier across the ranks (the
    device synchronised, then the group's barrier), so no kernel waits on
    another GPU's kernel:

      reduce    the local members' reduction into a scratch object
                (step 1), barrier, then b200shm_span_combine on every rank:
                the butterfly's cross-GPU levels over the G partials, read
                from the G arenas, fused with the write of the result to the
                local members' dest (steps 2 and 3 in one kernel), barrier
                (before the scratch is written again).  Long vectors go in
                chunks of the scratch's size.
      fcollect  barrier (every rank's source written), one kernel per rank
                reading every member's block from the GPU that holds it and
                writing the local members' dest, barrier (before any source
                is overwritten).
      alltoall  the same, each local member's dest blocks read from the
                members that hold them.
      amo       one-sided: system-scope atomics on the owner's arena, run
                by the calling GPU alone (no barrier, no exchange).

    Results are those of SpanningTeam: the same combine order, so the same
    bits (`exact`); byte-exact data movement; atomics exact.
    """

    def __init__(self, engine, members_per_rank, group=None, local_start=0, local_stride=1,
                 scratch_bytes=1 << 22):
        super().__init__(engine, members_per_rank, group, local_start, local_stride)
        G = self.world
        if not _pow2(G) or G > 16:
            raise ValueError("PeerTeam: %d ranks (a power of two up to 16)" % G)
        self.scratch_bytes = scratch_bytes
        self.scratch = engine.malloc(scratch_bytes)
        mine = (engine.ipc_handle(), engine.heap_slice(), engine.n_pes(), self.local,
                self.scratch)
        infos = [None] * G
        dist.all_gather_object(infos, mine, group=group)
        # every rank sees the same table, so every rank refuses together
        if len({(i[1], i[2], i[3]) for i in infos}) != 1:
            engine.free(self.scratch)
            raise ValueError("PeerTeam: every rank needs the same npes, heap size and local team")
        self.slice = mine[1]
        self.bases = [engine.heap_base() if r == self.rank else engine.peer_open(info[0])
                      for r, info in enumerate(infos)]
        self.scratch_of = [info[4] for info in infos]

    def barrier(self):
        self.sync_device()
        dist.barrier(group=self.group)

    def close(self):
        """Unmap the peers' arenas and free the scratch (all ranks together)."""
        self.barrier()
        for r, b in enumerate(self.bases):
            if r != self.rank:
                self.B.peer_close(b)
        self.B.free(self.scratch)
        self.bases = []
        dist.barrier(group=self.group)

    def reduce(self, op, dtype, algo, dest, src, nelems):
        """All-reduce over the spanning team; returns True when the result is
        bit-identical to the reference's (see `exact`)."""
        start, stride, L = self.local
        es = torch.empty((), dtype=_TORCH[dtype]).element_size() if dtype in _TORCH else \
            {"complex64": 8, "complex128": 16}[dtype]
        chunk = self.scratch_bytes // es
        partials = [self.bases[g] + start * self.slice + self.scratch_of[g]
                    for g in range(self.world)]
        e0 = 0
        while e0 < nelems:
            n = min(chunk, nelems - e0)
            self.B.reduce(op, dtype, algo, self.scratch, src + e0 * es, n, team=self.local)
            self.barrier()
            self.B.span_combine(op, dtype, self.world, self.rank, partials, dest + e0 * es, n,
                                team=self.local)
            self.barrier()
            e0 += n
        return self.exact(op, dtype, algo)

    def amo(self, amo, dtype, pe, off, value, cond=None):
        """One-sided atomics on (member, offset) targets anywhere in the
        team: this GPU runs every op as a system-scope atomic on the owner's
        arena (peer memory for members on other GPUs), with no exchange and
        no other rank taking part; returns the old values (int64, on the CPU,
        in the caller's order).  Ops of different ranks on one word are
        applied atomically in an unspecified order (src/shmemc/ucx/comms.c:
        409-671).  dtype: 4- or 8-byte."""
        wide = dtype in ("int64", "uint64", "float64")
        tdt = torch.int64 if wide else torch.int32
        n = len(pe)
        if n == 0:
            return torch.zeros(0, dtype=torch.int64)
        member = torch.as_tensor(pe, dtype=torch.int64).to(torch.int32).cuda()
        o = torch.as_tensor(off, dtype=torch.int64).cuda()
        v = torch.as_tensor(value, dtype=torch.int64).to(tdt).cuda()
        c = None if cond is None else torch.as_tensor(cond, dtype=torch.int64).to(tdt).cuda()
        f = torch.empty(n, dtype=tdt, device="cuda")  # written whole by the engine
        self.B.span_amo(amo, dtype, self.world, self.bases, n, member.data_ptr(), o.data_ptr(),
                        v.data_ptr(), None if c is None else c.data_ptr(), f.data_ptr(),
                        team=self.local)
        return f.cpu().to(torch.int64)

    def fcollect(self, dest, src, nbytes):
        """Every member's dest holds the P members' blocks in member order
        (fcollect_helper_*, src/shcoll/src/fcollect.c:32-484), each block
        read once from the GPU that holds it."""
        self.barrier()
        self.B.span_fcollect(self.world, self.rank, self.bases, dest, src, nbytes,
                             team=self.local)
        self.barrier()

    def alltoall(self, dest, src, nbytes):
        """Member j's dest block k = member k's source block j
        (alltoall_helper_*, src/shcoll/src/alltoall.c:75-201), read from
        whichever GPU holds member k."""
        self.barrier()
        self.B.span_alltoall(self.world, self.rank, self.bases, dest, src, nbytes,
                             team=self.local)
        self.barrier()


_TORCH = {"int8": torch.int8, "int16": torch.int16, "int32": torch.int32, "int64": torch.int64,
          "uint8": torch.uint8, "uint16": torch.uint16, "uint32": torch.uint32,
          "uint64": torch.uint64, "float32": torch.float32, "float64": torch.float64}
_TYPESTR = {"int8": "|i1", "int16": "<i2", "int32": "<i4", "int64": "<i8", "uint8": "|u1",
            "uint16": "<u2", "uint32": "<u4", "uint64": "<u8", "float32": "<f4",
            "float64": "<f8"}


class _DevArray:
    """A device buffer described by __cuda_array_interface__, so torch can
    view arena memory without copying."""

    def __init__(self, ptr, n, dtype):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": _TYPESTR[dtype],
                                         "data": (int(ptr), False), "version": 3}


def _device_tensor(ptr, n, dtype):
    return torch.as_tensor(_DevArray(ptr, n, dtype), device="cuda")
