"""ctypes access to the two CPU checkers.  TEST INFRASTRUCTURE ONLY.

* ``Restatement`` -- my plain-C restatement of the shcoll results
  (oracle/shcoll_oracle.c, built into oracle/_build/liboracle.so).  It is the
  checker the GPU parity tests use, because it builds from committed source
  anywhere.
* ``Reference`` -- the reference's own shcoll algorithm code
  (BTMichalowicz/osss-ucx src/shcoll/src/*.c) compiled unmodified and run
  over in-process emulated PEs (oracle/_ref/libref_shcoll.so).  It pins the
  restatement and is the timed CPU baseline.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "_build", "liboracle.so")
REFERENCE_SO = os.path.join(HERE, "_ref", "libref_shcoll.so")

# machine dtypes shared with the product's enum (osss-ucx_b200/csrc/b200shm_types.h)
DTYPES = ["int8", "int16", "int32", "int64", "uint8", "uint16", "uint32", "uint64",
          "float32", "float64", "float80", "complex64", "complex128"]
NP = {"int8": np.int8, "int16": np.int16, "int32": np.int32, "int64": np.int64,
      "uint8": np.uint8, "uint16": np.uint16, "uint32": np.uint32, "uint64": np.uint64,
      "float32": np.float32, "float64": np.float64, "float80": np.longdouble,
      "complex64": np.complex64, "complex128": np.complex128}
OPS = ["and", "or", "xor", "min", "max", "sum", "prod"]
ALGOS = ["linear", "binomial", "rec_dbl", "rabenseifner", "rabenseifner2"]

# OpenSHMEM type names (include/shmem/api_types.h) -> machine dtype on x86-64
SHMEM_TYPES = {
    "char": "int8", "schar": "int8", "short": "int16", "int": "int32", "long": "int64",
    "longlong": "int64", "ptrdiff": "int64", "uchar": "uint8", "ushort": "uint16",
    "uint": "uint32", "ulong": "uint64", "ulonglong": "uint64", "int8": "int8",
    "int16": "int16", "int32": "int32", "int64": "int64", "uint8": "uint8",
    "uint16": "uint16", "uint32": "uint32", "uint64": "uint64", "size": "uint64",
    "float": "float32", "double": "float64", "longdouble": "float80",
    "complexf": "complex64", "complexd": "complex128",
}
# type tables of api_types.h: which names exist per op class
REDUCE_BITWISE = ["uchar", "ushort", "uint", "ulong", "ulonglong", "int8", "int16",
                  "int32", "int64", "uint8", "uint16", "uint32", "uint64", "size"]
REDUCE_MINMAX = ["char", "schar", "short", "int", "long", "longlong", "ptrdiff", "uchar",
                 "ushort", "uint", "ulong", "ulonglong", "int8", "int16", "int32",
                 "int64", "uint8", "uint16", "uint32", "uint64", "size", "float",
                 "double", "longdouble"]
REDUCE_ARITH = REDUCE_MINMAX + ["complexd", "complexf"]
TO_ALL_BITWISE = ["short", "int", "long", "longlong"]
TO_ALL_MINMAX = ["short", "int", "long", "longlong", "float", "double", "longdouble"]
TO_ALL_ARITH = TO_ALL_MINMAX + ["complexd", "complexf"]


def reduce_types(op, form="reduce"):
    if form == "reduce":
        return REDUCE_BITWISE if op in ("and", "or", "xor") else (
            REDUCE_MINMAX if op in ("min", "max") else REDUCE_ARITH)
    return TO_ALL_BITWISE if op in ("and", "or", "xor") else (
        TO_ALL_MINMAX if op in ("min", "max") else TO_ALL_ARITH)


def reference_tree():
    """The reference source tree: $REFERENCE_TREE, else a `reference`
    directory beside this repository; None when neither exists."""
    cand = os.environ.get("REFERENCE_TREE") or os.path.join(
        os.path.dirname(os.path.dirname(HERE)), "reference")
    return cand if os.path.isfile(os.path.join(cand, "src", "shcoll", "src", "reduce.c")) else None


def build(reference=True):
    """Compile the restatement and, when the reference tree is found, _ref."""
    tree = reference_tree() if reference else None
    cmd = ["make", "-s", "-C", HERE, "all" if tree else "restatement"]
    if tree:
        cmd.append("REF=" + tree)
    subprocess.run(cmd, check=True)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


class Restatement:
    """My CPU restatement (oracle/shcoll_oracle.c)."""

    def __init__(self, path=RESTATEMENT_SO):
        if not os.path.exists(path):
            build(reference=False)
        L = ctypes.CDLL(path)
        vp, sz, ci = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
        L.or_reduce.argtypes = [ci, ci, ci, ci, sz, vp, vp]
        L.or_fcollect.argtypes = [ci, sz, vp, vp]
        L.or_alltoall.argtypes = [ci, sz, vp, vp]
        L.or_alltoalls.argtypes = [ci, sz, ctypes.c_long, ctypes.c_long, sz, vp, vp]
        L.or_broadcast.argtypes = [ci, ci, sz, vp, vp]
        L.or_amo_fetch_add_i64.argtypes = [ci, sz, sz, vp, vp, vp, vp, vp]
        L.or_reverse_bits.argtypes = [ci, ci]
        self.L = L

    def reduce(self, algo, op, x):
        """x: [P, N] member-ordered inputs of a numpy dtype; returns [P, N]."""
        x = np.ascontiguousarray(x)
        dt = _dtype_name(x.dtype)
        out = np.empty_like(x)
        rc = self.L.or_reduce(ALGOS.index(algo), OPS.index(op), DTYPES.index(dt),
                              x.shape[0], x.shape[1], _ptr(x), _ptr(out))
        if rc != 0:
            raise ValueError(f"oracle reduce rejected {algo}/{op}/{dt}")
        return out

    def fcollect(self, x):
        x = np.ascontiguousarray(x)
        P = x.shape[0]
        out = np.empty((P, x.size), dtype=x.dtype)
        self.L.or_fcollect(P, x[0].nbytes, _ptr(x), _ptr(out))
        return out

    def collect(self, x, nbytes, dest_bytes):
        """x: [P, >= max(nbytes)] uint8 rows; member k contributes nbytes[k];
        returns [P, dest_bytes] uint8 with the concatenation first."""
        x = np.ascontiguousarray(x, dtype=np.uint8)
        P = x.shape[0]
        nb = np.ascontiguousarray(nbytes, dtype=np.uint64)
        out = np.zeros((P, dest_bytes), dtype=np.uint8)
        rc = self.L.or_collect(P, _ptr(nb), _ptr(x), ctypes.c_size_t(x.shape[1]), _ptr(out),
                               ctypes.c_size_t(dest_bytes))
        if rc != 0:
            raise ValueError("oracle collect rejected its sizes")
        return out

    def alltoall(self, x):
        """x: [P, P*n]: row k is member k's source (P blocks)."""
        x = np.ascontiguousarray(x)
        P = x.shape[0]
        out = np.empty_like(x)
        self.L.or_alltoall(P, x[0].nbytes // P, _ptr(x), _ptr(out))
        return out

    def alltoalls(self, x, dest_init, dst, sst, nelems):
        x = np.ascontiguousarray(x)
        out = np.array(dest_init, copy=True, order="C")
        self.L.or_alltoalls(x.shape[0], nelems, dst, sst, x.itemsize, _ptr(x), _ptr(out))
        return out

    def broadcast(self, x, dest_init, root):
        x = np.ascontiguousarray(x)
        out = np.array(dest_init, copy=True, order="C")
        self.L.or_broadcast(x.shape[0], root, x[0].nbytes, _ptr(x), _ptr(out))
        return out

    def amo_fetch_add(self, npes, ncounters, pe, off, val, counters):
        pe = np.ascontiguousarray(pe, dtype=np.int32)
        off = np.ascontiguousarray(off, dtype=np.int64)
        val = np.ascontiguousarray(val, dtype=np.int64)
        c = np.array(counters, dtype=np.int64, copy=True)
        fetched = np.empty(len(pe), dtype=np.int64)
        rc = self.L.or_amo_fetch_add_i64(npes, ncounters, len(pe), _ptr(pe), _ptr(off),
                                         _ptr(val), _ptr(fetched), _ptr(c))
        if rc != 0:
            raise ValueError("bad AMO target")
        return fetched, c


def _dtype_name(dt):
    dt = np.dtype(dt)
    for k, v in NP.items():
        if np.dtype(v) == dt:
            return k
    raise TypeError(dt)


# job kinds understood by ref_run (oracle/ref_harness/pe_emu.c)
K_REDUCE_TEAM, K_TO_ALL, K_SIZED, K_TEAM_COPY, K_ALLTOALLS_SIZED, K_ALLTOALLS_TEAM, \
    K_BARRIER, K_BARRIER_ALL, K_TEAM_SYNC, K_BROADCAST_SIZED, K_BROADCAST_TEAM, \
    K_COLLECT_SIZED, K_COLLECT_TEAM = range(13)


class Reference:
    """The reference's own shcoll code over emulated PEs (oracle/_ref)."""

    available = os.path.exists(REFERENCE_SO)

    def __init__(self, path=REFERENCE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (build with `make -C oracle reference`)")
        L = ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)
        ci, sz, vp, cl = ctypes.c_int, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_long
        L.ref_run.argtypes = [ci, ctypes.c_char_p, ci, ci, ci, ci, sz, cl, cl, vp, sz, vp,
                              sz, ci, ci, vp, ci]
        L.ref_set_wait_limit.argtypes = [ctypes.c_double]
        self.L = L

    def run(self, kind, fname, x, out, npes=None, pe_start=0, log_stride=0, nelems=0,
            a=0, b=0, warmup=0, iters=1, pin=False):
        """x: [pe_size, src_bytes-shaped], out: [pe_size, ...] initial dest, updated."""
        P = x.shape[0]
        npes = npes or pe_start + (P - 1) * (1 << log_stride) + 1
        times = np.zeros(iters, dtype=np.float64)
        rc = self.L.ref_run(kind, fname.encode(), npes, pe_start, log_stride, P, nelems,
                            a, b, _ptr(x), x[0].nbytes if x.size else 0, _ptr(out),
                            out[0].nbytes if out.size else 0, warmup, iters, _ptr(times),
                            int(pin))
        if rc != 0:
            raise RuntimeError(f"ref_run({fname}) failed rc={rc}")
        return out, times

    def reduce(self, algo, op, x, tname=None, form="team", **kw):
        x = np.ascontiguousarray(x)
        tname = tname or {"int8": "int8", "int16": "int16", "int32": "int32",
                          "int64": "int64", "uint8": "uint8", "uint16": "uint16",
                          "uint32": "uint32", "uint64": "uint64", "float32": "float",
                          "float64": "double", "float80": "longdouble",
                          "complex64": "complexf", "complex128": "complexd"}[_dtype_name(x.dtype)]
        out = np.zeros_like(x)
        if form == "team":
            return self.run(K_REDUCE_TEAM, f"shcoll_{tname}_{op}_reduce_{algo}", x, out,
                            nelems=x.shape[1], **kw)
        return self.run(K_TO_ALL, f"shcoll_{tname}_{op}_to_all_{algo}", x, out,
                        nelems=x.shape[1], **kw)
