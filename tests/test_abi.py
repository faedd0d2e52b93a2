"""The C ABI library loads on any machine and exports every entry point its
public headers declare; without a GPU every compute call fails cleanly."""
import ctypes
import os
import re

import b200shm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in sorted(os.listdir(os.path.join(ROOT, "include")))
           if h.startswith("b200shm") and h.endswith(".h")]


def declared(header):
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(b200shm_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    assert HEADERS
    lib = ctypes.CDLL(b200shm.LIB_PATH)
    missing = []
    for h in HEADERS:
        for name in declared(h):
            try:
                getattr(lib, name)
            except AttributeError:
                missing.append((os.path.basename(h), name))
    assert not missing, missing


def test_calls_before_init_fail_with_state_error():
    L = b200shm.lib
    if L.b200shm_initialized():
        return  # a GPU session already initialised the engine in this process
    rc = L.b200shm_reduce(5, 8, 2, 0, 1, 4, 0, 0, 16, None)
    assert rc == -5 and b"not initialised" in L.b200shm_last_error()
    assert L.b200shm_fcollect(0, 1, 4, 0, 0, 64, None) == -5
    assert L.b200shm_barrier(2, 0, 1, 4, None) == -5
    assert L.b200shm_ptr(0, 0) is None
    # the span calls check the team (and so the engine) before any address
    addrs = (ctypes.c_uint64 * 2)(1 << 40, 1 << 41)
    assert L.b200shm_span_fcollect(2, 0, addrs, 0, 1, 4, 0, 0, 64, None) == -5
    assert L.b200shm_span_alltoall(2, 0, addrs, 0, 1, 4, 0, 0, 64, None) == -5
    assert L.b200shm_span_combine(5, 8, 2, 0, addrs, 0, 1, 4, 0, 16, None) == -5
    assert L.b200shm_span_amo(0, 3, 2, addrs, 0, 1, 4, 0, None, None, None, None, None,
                              None) == -5
    assert b"not initialised" in L.b200shm_last_error()
    # a bad rank count or rank is refused first, engine or not
    assert L.b200shm_span_fcollect(3, 0, addrs, 0, 1, 4, 0, 0, 64, None) == -1
    assert L.b200shm_span_alltoall(2, 2, addrs, 0, 1, 4, 0, 0, 64, None) == -1


def test_shmem_surface_exports_every_declared_function():
    """Every function include/shmem.h and include/shmemx.h declare (after
    macro expansion) is exported by libshmem_b200.so."""
    import subprocess
    import __graft_entry__
    __graft_entry__.build_library()
    host_lib = os.path.join(ROOT, "osss-ucx_b200", "lib", "libshmem_b200.so")
    text = subprocess.run(["gcc", "-E", "-P", "-x", "c", "-"], input='#include "shmemx.h"\n',
                          capture_output=True, text=True, check=True,
                          cwd=os.path.join(ROOT, "include")).stdout
    names = set(re.findall(r"\b((?:shmem|shmemx)_[a-z0-9_]+)\s*\(", text))
    assert len(names) > 600
    lib = ctypes.CDLL(host_lib)
    missing = sorted(n for n in names if not hasattr(lib, n))
    assert not missing, missing[:20]


def test_every_openshmem_declaration_is_exported():
    """include/shmem.h and shmemx.h generate most of their declarations from
    type tables; every function they declare (after the preprocessor) is
    exported by libshmem_b200.so."""
    import subprocess
    lib = ctypes.CDLL(os.path.join(ROOT, "osss-ucx_b200", "lib", "libshmem_b200.so"))
    missing = []
    for h in ("shmem.h", "shmemx.h"):
        text = subprocess.run(["gcc", "-E", "-P", "-x", "c", os.path.join(ROOT, "include", h)],
                              capture_output=True, text=True, check=True).stdout
        names = sorted(set(re.findall(r"\b((?:shmem|shmemx|pshmem)_[A-Za-z0-9_]+)\s*\(", text)))
        assert len(names) > (1000 if h == "shmem.h" else 4)
        for name in names:
            try:
                getattr(lib, name)
            except AttributeError:
                missing.append((h, name))
    assert not missing, missing[:20]


def test_noalloc_row_overlap_rules_without_a_gpu():
    """b200shm_reduce_noalloc checks its rows before it touches the device:
    interleaved rows (dest and source rows of different offsets in the same
    slices) and in-place rows pass the checks, any dest row that touches
    another member's source row is refused.  Without a GPU a call that
    passes the checks stops at the device (a CUDA error), so the code tells
    which way the check went.  Skipped where a GPU is present, since there
    a call that passes would run on these made-up addresses."""
    import torch
    if torch.cuda.is_available():
        return
    L = b200shm.lib
    base, sb, n = 1 << 40, 1 << 20, 256  # int32 rows of 1 KiB in slices of 1 MiB

    def call(dst, ds, src, ss, P=4):
        return L.b200shm_reduce_noalloc(5, 2, 2, P, dst, ds, src, ss, n, None)
    assert call(base + 4096, sb, base, sb) == -4          # interleaved: checks pass
    assert call(base, sb, base, sb) == -4                 # in place: checks pass
    assert call(base + 8 * sb, 2 * sb, base, sb) == -4    # apart, other stride
    for dst, ds, src, ss in [(base + sb + 4, sb, base, sb), (base, sb, base, 2 * sb),
                             (base + 64, sb, base, sb), (base + 3 * sb - 512, sb, base, sb)]:
        assert call(dst, ds, src, ss) == -1, (dst - base, ds, ss)
        assert b"overlaps" in L.b200shm_last_error()
