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

Step 2 moves N elements per round over NCCL (point-to-point over NVLink);
no TMA multicast is used anywhere on this path.  Nothing here has run on
more than one GPU: this pool gives one GPU per job, so the cross-rank
steps are exercised with gloo ranks on the CPU (tests/test_spanning_team.py).
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
