"""Python binding of the C ABI in include/b200shm.h (ctypes).

This is how the tests and the benchmark drive the engine: every call goes
through libb200shm.so.  There is no fallback of any kind -- if the library
cannot be loaded, importing this module raises.

Usage:
    import b200shm as B
    B.init(npes=64, heap_bytes=64 << 20)
    src = B.malloc(N * 4); dst = B.malloc(N * 4)
    B.put_rows(src, x)                      # x: [npes, N] numpy array
    B.reduce("sum", "float32", "rec_dbl", dst, src, N, team=(0, 1, 64))
    y = B.get_rows(dst, N * 4, np.float32, team=(0, 1, 64))
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libb200shm.so")

DTYPES = ["int8", "int16", "int32", "int64", "uint8", "uint16", "uint32", "uint64",
          "float32", "float64", "float80", "complex64", "complex128"]
OPS = ["and", "or", "xor", "min", "max", "sum", "prod"]
ALGOS = ["linear", "binomial", "rec_dbl", "rabenseifner", "rabenseifner2"]
BARRIER_ALGOS = ["linear", "complete_tree", "binomial_tree", "knomial_tree", "dissemination"]
AMOS = ["fetch_add", "add", "fetch_inc", "inc", "swap", "cswap", "set", "fetch", "fetch_and",
        "and", "fetch_or", "or", "fetch_xor", "xor"]
SERVE_ALLOC = (1 << 64) - 1  # request dest_off: the serving loop allocates the dest
STATUS = {0: "OK", -1: "ERR_ARG", -2: "ERR_UNSUPPORTED", -3: "ERR_NOMEM", -4: "ERR_CUDA",
          -5: "ERR_STATE", -6: "ERR_TIMEOUT", -7: "ERR_BUSY"}


class B200Error(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(LIB_PATH + " is missing: build it with `python osss-ucx_b200/build.py`")
    L = ctypes.CDLL(LIB_PATH)
    ci, u64, i64, vp = ctypes.c_int, ctypes.c_uint64, ctypes.c_int64, ctypes.c_void_p
    sig = {
        "b200shm_init": (ci, [ci, u64, ci]),
        "b200shm_finalize": (ci, []),
        "b200shm_initialized": (ci, []),
        "b200shm_n_pes": (ci, []),
        "b200shm_heap_slice": (u64, []),
        "b200shm_heap_base": (vp, []),
        "b200shm_ptr": (vp, [ci, u64]),
        "b200shm_last_error": (ctypes.c_char_p, []),
        "b200shm_quiet": (ci, []),
        "b200shm_launch_count": (ctypes.c_ulonglong, []),
        "b200shm_stream": (vp, []),
        "b200shm_malloc": (ci, [u64, u64, ctypes.POINTER(u64)]),
        "b200shm_free": (ci, [u64]),
        "b200shm_heap_free_bytes": (u64, []),
        "b200shm_put_host": (ci, [ci, ci, ci, u64, vp, u64, vp]),
        "b200shm_get_host": (ci, [vp, ci, ci, ci, u64, u64, vp]),
        "b200shm_memset": (ci, [ci, ci, ci, u64, ci, u64, vp]),
        "b200shm_reduce": (ci, [ci, ci, ci, ci, ci, ci, u64, u64, u64, vp]),
        "b200shm_reduce_noalloc": (ci, [ci, ci, ci, ci, vp, u64, vp, u64, u64, vp]),
        "b200shm_reduce_host": (ci, [ci, ci, ci, ci, ci, ci, vp, u64, vp, u64, u64, u64, u64, vp]),
        "b200shm_fcollect": (ci, [ci, ci, ci, u64, u64, u64, vp]),
        "b200shm_alltoall": (ci, [ci, ci, ci, u64, u64, u64, vp]),
        "b200shm_collect": (ci, [ci, ci, ci, u64, u64, vp, vp]),
        "b200shm_alltoalls": (ci, [ci, ci, ci, u64, u64, i64, i64, u64, u64, vp]),
        "b200shm_broadcast": (ci, [ci, ci, ci, ci, u64, u64, u64, vp]),
        "b200shm_barrier": (ci, [ci, ci, ci, ci, vp]),
        "b200shm_set_wait_budget": (u64, [u64]),
        "b200shm_barrier_absent": (ci, [ci, ci, ci, ci, ci, vp]),
        "b200shm_barrier_flags_nonzero": (i64, []),
        "b200shm_amo_batch": (ci, [ci, ci, u64, vp, vp, vp, vp, vp, vp]),
        "b200shm_batch_create": (ci, [vp, u64, ci, ctypes.POINTER(vp)]),
        "b200shm_batch_run": (ci, [vp, vp]),
        "b200shm_batch_destroy": (ci, [vp]),
        "b200shm_reduce_batch": (ci, [vp, u64, vp]),
        "b200shm_fill_uniform": (ci, [ci, ci, ci, u64, ci, u64, u64, ctypes.c_double,
                                      ctypes.c_double, vp]),
        "b200shm_serve_start": (ci, [ctypes.c_uint32, ci, ctypes.c_double, ctypes.POINTER(vp)]),
        "b200shm_serve_start_budget": (ci, [ctypes.c_uint32, ci, ctypes.c_double, u64,
                                            ctypes.POINTER(vp)]),
        "b200shm_serve_enqueue": (ci, [vp, vp, ctypes.POINTER(u64)]),
        "b200shm_serve_poll": (ci, [vp, u64, ctypes.POINTER(u64)]),
        "b200shm_serve_wait": (ci, [vp, u64, ctypes.c_double, ctypes.POINTER(u64)]),
        "b200shm_serve_stop": (ci, [vp]),
        "b200shm_serve_trace": (ci, [vp, u64, vp]),
        "b200shm_serve_replay": (ci, [vp, vp, u64, vp, vp, vp]),
        "b200shm_serve_replay_ordered": (ci, [vp, u64, vp, ctypes.POINTER(ctypes.c_double), vp]),
        "b200shm_amo": (ci, [ci, ci, ci, u64, vp, vp, vp]),
        "b200shm_ipc_handle": (ci, [vp]),
        "b200shm_peer_open": (ci, [vp, ctypes.POINTER(vp)]),
        "b200shm_peer_close": (ci, [vp]),
        "b200shm_span_combine": (ci, [ci, ci, ci, ci, vp, ci, ci, ci, u64, u64, vp]),
        "b200shm_span_fcollect": (ci, [ci, ci, vp, ci, ci, ci, u64, u64, u64, vp]),
        "b200shm_span_alltoall": (ci, [ci, ci, vp, ci, ci, ci, u64, u64, u64, vp]),
        "b200shm_span_amo": (ci, [ci, ci, ci, vp, ci, ci, ci, u64, vp, vp, vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


lib = _load()


def _check(rc):
    if rc != 0:
        raise B200Error(rc, lib.b200shm_last_error().decode())
    return rc


def _team(team):
    if team is None:
        return 0, 1, lib.b200shm_n_pes()
    return team


def init(npes, heap_bytes, managed=False):
    return _check(lib.b200shm_init(npes, heap_bytes, 1 if managed else 0))


def finalize():
    return _check(lib.b200shm_finalize())


def initialized():
    return bool(lib.b200shm_initialized())


def n_pes():
    return lib.b200shm_n_pes()


def malloc(nbytes, align=256):
    off = ctypes.c_uint64(0)
    _check(lib.b200shm_malloc(nbytes, align, ctypes.byref(off)))
    return off.value


def free(off):
    return _check(lib.b200shm_free(off))


def launch_count():
    """Kernels launched by libb200shm.so since it was loaded."""
    return lib.b200shm_launch_count()


def stream():
    """The library stream (a cudaStream_t as an int)."""
    return lib.b200shm_stream()


def quiet():
    return _check(lib.b200shm_quiet())


def ptr(pe, off):
    return lib.b200shm_ptr(pe, off)


def put_rows(off, x, team=None, stream=None):
    """Copy host rows x[i] into member i's slice at `off`."""
    start, stride, size = _team(team)
    x = np.ascontiguousarray(x)
    assert x.shape[0] == size
    return _check(lib.b200shm_put_host(start, stride, size, off, x.ctypes.data,
                                       x[0].nbytes if size else 0, stream))


def get_rows(off, row_bytes, dtype, team=None, stream=None, out=None):
    """Copy row_bytes at `off` of every member into a host [size, ...] array."""
    start, stride, size = _team(team)
    dt = np.dtype(dtype)
    if out is None:
        out = np.empty((size, row_bytes // dt.itemsize), dtype=dt)
    _check(lib.b200shm_get_host(out.ctypes.data, start, stride, size, off, row_bytes, stream))
    return out


def memset(off, byte, nbytes, team=None, stream=None):
    start, stride, size = _team(team)
    return _check(lib.b200shm_memset(start, stride, size, off, byte, nbytes, stream))


def reduce(op, dtype, algo, dest, src, nelems, team=None, stream=None):
    start, stride, size = _team(team)
    return _check(lib.b200shm_reduce(OPS.index(op), DTYPES.index(dtype), ALGOS.index(algo),
                                     start, stride, size, dest, src, nelems, stream))


def reduce_host(op, dtype, algo, dest, src, x, out=None, team=None, stream=None):
    """All-reduce of host rows x[i] (member i) through the objects at src/dest;
    returns (or fills) the host result rows.  Pinned arrays let the copies overlap."""
    start, stride, size = _team(team)
    x = np.ascontiguousarray(x)
    if out is None:
        out = np.empty_like(x)
    _check(lib.b200shm_reduce_host(OPS.index(op), DTYPES.index(dtype), ALGOS.index(algo), start,
                                   stride, size, out.ctypes.data, out[0].nbytes, x.ctypes.data,
                                   x[0].nbytes, dest, src, x.shape[1], stream))
    return out


def reduce_noalloc(op, dtype, algo, npes, dest_ptr, dest_stride, src_ptr, src_stride, nelems,
                   stream=None):
    """All-reduce over caller-owned device buffers (device addresses as ints);
    allocates nothing and needs no init()."""
    return _check(lib.b200shm_reduce_noalloc(OPS.index(op), DTYPES.index(dtype),
                                             ALGOS.index(algo), npes, dest_ptr, dest_stride,
                                             src_ptr, src_stride, nelems, stream))


def fcollect(dest, src, nbytes, team=None, stream=None):
    start, stride, size = _team(team)
    return _check(lib.b200shm_fcollect(start, stride, size, dest, src, nbytes, stream))


def collect(dest, src, nbytes, team=None, stream=None):
    """Variable-size allgather: member k contributes nbytes[k] bytes."""
    start, stride, size = _team(team)
    nb = np.ascontiguousarray(nbytes, dtype=np.uint64)
    if len(nb) != size:
        raise ValueError("one size per member")
    return _check(lib.b200shm_collect(start, stride, size, dest, src, nb.ctypes.data, stream))


def alltoall(dest, src, nbytes, team=None, stream=None):
    start, stride, size = _team(team)
    return _check(lib.b200shm_alltoall(start, stride, size, dest, src, nbytes, stream))


def alltoalls(dest, src, dst, sst, nelems, elem_size, team=None, stream=None):
    start, stride, size = _team(team)
    return _check(lib.b200shm_alltoalls(start, stride, size, dest, src, dst, sst, nelems,
                                        elem_size, stream))


def heap_slice():
    return lib.b200shm_heap_slice()


def heap_base():
    """Device address of slice 0 of this process's arena."""
    return lib.b200shm_heap_base() or 0


def ipc_handle():
    """The arena's CUDA IPC handle (64 bytes) for another process to map."""
    h = ctypes.create_string_buffer(64)
    _check(lib.b200shm_ipc_handle(h))
    return h.raw


def peer_open(handle):
    """Map another process's arena; returns the device address of its slice 0."""
    base = ctypes.c_void_p()
    _check(lib.b200shm_peer_open(bytes(handle), ctypes.byref(base)))
    return base.value


def peer_close(base):
    return _check(lib.b200shm_peer_close(base))


def _addrs(addrs):
    a = np.ascontiguousarray(addrs, dtype=np.uint64)
    return a, a.ctypes.data


def span_combine(op, dtype, G, rank, partials, dest, nelems, team=None, stream=None):
    """The cross-GPU butterfly levels over G partial vectors at the device
    addresses `partials`, written to this GPU's team members at `dest`."""
    start, stride, size = _team(team)
    a, ap = _addrs(partials)
    return _check(lib.b200shm_span_combine(OPS.index(op), DTYPES.index(dtype), G, rank, ap, start,
                                           stride, size, dest, nelems, stream))


def span_fcollect(G, rank, bases, dest, src, nbytes, team=None, stream=None):
    start, stride, size = _team(team)
    a, ap = _addrs(bases)
    return _check(lib.b200shm_span_fcollect(G, rank, ap, start, stride, size, dest, src, nbytes,
                                            stream))


def span_alltoall(G, rank, bases, dest, src, nbytes, team=None, stream=None):
    start, stride, size = _team(team)
    a, ap = _addrs(bases)
    return _check(lib.b200shm_span_alltoall(G, rank, ap, start, stride, size, dest, src, nbytes,
                                            stream))


def span_amo(amo, dtype, G, bases, nops, member_dev, off_dev, value_dev=None, cond_dev=None,
             fetched_dev=None, team=None, stream=None):
    """One-sided atomics on any member of a spanning team (device arrays:
    int32 members, uint64 byte offsets, 4- or 8-byte operands)."""
    start, stride, size = _team(team)
    a, ap = _addrs(bases)
    return _check(lib.b200shm_span_amo(AMOS.index(amo), DTYPES.index(dtype), G, ap, start, stride,
                                       size, nops, member_dev, off_dev, value_dev, cond_dev,
                                       fetched_dev, stream))


def broadcast(root, dest, src, nbytes, team=None, stream=None):
    start, stride, size = _team(team)
    return _check(lib.b200shm_broadcast(root, start, stride, size, dest, src, nbytes, stream))


def barrier(algo="binomial_tree", team=None, stream=None):
    start, stride, size = _team(team)
    return _check(lib.b200shm_barrier(BARRIER_ALGOS.index(algo), start, stride, size, stream))


def set_wait_budget(seconds):
    """Budget of every device barrier wait (0 = the default 2 s); returns the
    previous budget in seconds."""
    return lib.b200shm_set_wait_budget(int(seconds * 1e9)) * 1e-9


def barrier_absent(algo, absent, team=None, stream=None):
    """Barrier with member `absent` never arriving (failure injection)."""
    start, stride, size = _team(team)
    return _check(lib.b200shm_barrier_absent(BARRIER_ALGOS.index(algo), start, stride, size,
                                             absent, stream))


def barrier_flags_nonzero():
    n = lib.b200shm_barrier_flags_nonzero()
    if n < 0:
        _check(n)
    return n


def amo_batch(amo, dtype, nops, pe_dev, off_dev, value_dev=None, cond_dev=None,
              fetched_dev=None, stream=None):
    """Device-array AMO batch; *_dev are device addresses (ints)."""
    return _check(lib.b200shm_amo_batch(AMOS.index(amo), DTYPES.index(dtype), nops, pe_dev,
                                        off_dev, value_dev, cond_dev, fetched_dev, stream))


# ---------------------------------------------------------------------------
# batched reductions
# ---------------------------------------------------------------------------
BATCH_NO_TUNE = 0x1
BATCH_GRAPH = 0x2
BATCH_TUNE = 0x4


class ReduceDesc(ctypes.Structure):
    """b200shm_reduce_desc"""
    _fields_ = [("op", ctypes.c_int32), ("dtype", ctypes.c_int32), ("algo", ctypes.c_int32),
                ("pe_start", ctypes.c_int32), ("pe_stride", ctypes.c_int32),
                ("pe_size", ctypes.c_int32), ("dest_off", ctypes.c_uint64),
                ("src_off", ctypes.c_uint64), ("nelems", ctypes.c_uint64),
                ("lanes", ctypes.c_int32), ("tile", ctypes.c_int32)]


def make_descs(items):
    """items: dicts with op, dtype, algo ("auto" allowed), team=(start, stride, size),
    dest, src, nelems."""
    arr = (ReduceDesc * len(items))()
    for i, it in enumerate(items):
        start, stride, size = it["team"]
        algo = it.get("algo", "rec_dbl")
        arr[i] = ReduceDesc(OPS.index(it["op"]), DTYPES.index(it["dtype"]),
                            -1 if algo == "auto" else ALGOS.index(algo), start, stride, size,
                            it["dest"], it["src"], it["nelems"], 0, 0)
    return arr


class Batch:
    """A planned batch of independent reductions (b200shm_batch_create / run / destroy)."""

    def __init__(self, descs, flags=0):
        self.descs = descs
        self.h = None
        h = ctypes.c_void_p()
        _check(lib.b200shm_batch_create(ctypes.cast(descs, ctypes.c_void_p), len(descs), flags,
                                        ctypes.byref(h)))
        self.h = h

    def run(self, stream=None):
        return _check(lib.b200shm_batch_run(self.h, stream))

    def close(self):
        if self.h and lib is not None:  # lib is None during interpreter teardown
            lib.b200shm_batch_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()


def fill_uniform(off, dtype, nelems, seed, lo, hi, team=None, stream=None):
    """Seeded uniform values at `off` in every member (ints in [lo, hi], floats in [lo, hi))."""
    start, stride, size = _team(team)
    return _check(lib.b200shm_fill_uniform(start, stride, size, off, DTYPES.index(dtype), nelems,
                                           seed, lo, hi, stream))


# ---------------------------------------------------------------------------
# serving loop
# ---------------------------------------------------------------------------
REQ_KINDS = ["reduce", "fcollect", "alltoall", "put", "get", "amo"]


class Request(ctypes.Structure):
    """b200shm_request"""
    _fields_ = [("kind", ctypes.c_int32), ("op", ctypes.c_int32), ("dtype", ctypes.c_int32),
                ("algo", ctypes.c_int32), ("pe_start", ctypes.c_int32),
                ("pe_stride", ctypes.c_int32), ("pe_size", ctypes.c_int32),
                ("pe", ctypes.c_int32), ("dest_off", ctypes.c_uint64),
                ("src_off", ctypes.c_uint64), ("n", ctypes.c_uint64),
                ("value", ctypes.c_uint64), ("cond", ctypes.c_uint64)]


def make_requests(items):
    """items: dicts with kind and the fields it uses: op (a reduce op name, or
    an AMO name for kind "amo"), dtype, algo, team=(start, stride, size),
    pe, dest, src, n, value, cond."""
    arr = (Request * len(items))()
    for i, it in enumerate(items):
        kind = it["kind"]
        start, stride, size = it.get("team", (0, 1, 1))
        op = it.get("op", "sum")
        opi = AMOS.index(op) if kind == "amo" else OPS.index(op)
        algo = it.get("algo", "rec_dbl")
        arr[i] = Request(REQ_KINDS.index(kind), opi, DTYPES.index(it.get("dtype", "int64")),
                         -1 if algo == "auto" else ALGOS.index(algo), start, stride, size,
                         it.get("pe", 0), it.get("dest", 0), it.get("src", 0), it.get("n", 0),
                         it.get("value", 0) & (2 ** 64 - 1), it.get("cond", 0) & (2 ** 64 - 1))
    return arr


class Server:
    """The serving loop (b200shm_serve_start / enqueue / poll / wait / stop)."""

    def __init__(self, queue_slots=1024, ctas=0, idle_seconds=0.25, heap_budget=0):
        """heap_budget: symmetric-heap bytes that admitted, incomplete
        requests may write at once (0 = no limit)."""
        h = ctypes.c_void_p()
        _check(lib.b200shm_serve_start_budget(queue_slots, ctas, idle_seconds, heap_budget,
                                              ctypes.byref(h)))
        self.h = h

    def enqueue(self, req):
        t = ctypes.c_uint64()
        _check(lib.b200shm_serve_enqueue(self.h, ctypes.byref(req), ctypes.byref(t)))
        return t.value

    def poll(self, ticket):
        f = ctypes.c_uint64()
        rc = lib.b200shm_serve_poll(self.h, ticket, ctypes.byref(f))
        if rc < 0:
            _check(rc)
        return (rc == 1), f.value

    def wait(self, ticket, timeout=30.0):
        f = ctypes.c_uint64()
        _check(lib.b200shm_serve_wait(self.h, ticket, timeout, ctypes.byref(f)))
        return f.value

    def trace(self, ticket):
        """Device times in ns (copied to the device, last claimed, done), or None."""
        t = np.zeros(3, np.uint64)
        if lib.b200shm_serve_trace(self.h, ticket, t.ctypes.data) != 1:
            return None
        return [int(v) for v in t]

    def replay(self, reqs, arrival_s):
        return replay(reqs, arrival_s, self)

    def stop(self):
        if self.h and lib is not None:
            _check(lib.b200shm_serve_stop(self.h))
        self.h = None

    def __del__(self):
        if getattr(self, "h", None):
            try:
                self.stop()
            except Exception:
                pass


def replay(reqs, arrival_s, server=None):
    """Open-loop replay: returns (latency seconds per request, fetched values)."""
    n = len(reqs)
    arr = np.ascontiguousarray(arrival_s, dtype=np.float64)
    lat = np.zeros(n, np.float64)
    fet = np.zeros(n, np.uint64)
    _check(lib.b200shm_serve_replay(server.h if server else None, ctypes.cast(reqs, ctypes.c_void_p),
                                    n, arr.ctypes.data, lat.ctypes.data, fet.ctypes.data))
    return lat, fet


def replay_ordered(reqs, stream=None):
    """Every request through its per-call entry point, stream-ordered, one
    synchronisation at the end: returns (seconds, fetched values)."""
    if not isinstance(reqs, ctypes.Array):  # e.g. a slice of an array: a list of requests
        reqs = (Request * len(reqs))(*reqs)
    n = len(reqs)
    fet = np.zeros(n, np.uint64)
    sec = ctypes.c_double()
    _check(lib.b200shm_serve_replay_ordered(ctypes.cast(reqs, ctypes.c_void_p), n, stream,
                                            ctypes.byref(sec), fet.ctypes.data))
    return sec.value, fet
