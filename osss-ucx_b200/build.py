"""Build libb200shm.so (the CUDA engine behind include/b200shm.h) in-tree.

    python osss-ucx_b200/build.py         # incremental
    python osss-ucx_b200/build.py --clean

Every translation unit is compiled for sm_100a only; objects go to
osss-ucx_b200/_build/, the library to osss-ucx_b200/lib/.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "lib")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                  "--expt-relaxed-constexpr", "-I" + INCLUDE, "-I" + CSRC]
CUDA_LIB = "libb200shm.so"
HOST_LIB = "libshmem_b200.so"
CC = os.environ.get("CC", "gcc")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    return hs + [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]


def _compile(src, obj, extra=()):
    cmd = [NVCC] + NVFLAGS + list(extra) + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
    return obj


def build(verbose=False, extra=()):
    """Compile every .cu under csrc/ and link lib/libb200shm.so; returns its path."""
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIB, exist_ok=True)
    heads = _headers()
    # the long double reduce units (software x87 arithmetic in every
    # instantiation) take far longer than the rest: start them first
    srcs = sorted((os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu")),
                  key=lambda p: (not os.path.basename(p).startswith("reduce_f80_"), p))
    lib = os.path.join(LIB, CUDA_LIB)
    if not extra and not _stale(lib, srcs + heads + [__file__]):
        build_host(lib)
        return lib  # up to date (objects may be absent, e.g. in a shipped snapshot)
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if _stale(o, [s] + heads + [__file__]):
            jobs.append((s, o))
    workers = max(8, os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(max_workers=min(workers, len(jobs) or 1)) as ex:
        for o in ex.map(lambda so: _compile(so[0], so[1], extra), jobs):
            if verbose:
                print("compiled", o)
    if _stale(lib, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    build_host(lib)
    return lib


def build_host(cuda_lib=None):
    """The OpenSHMEM surface (include/shmem.h) in C over libb200shm.so."""
    cuda_lib = cuda_lib or os.path.join(LIB, CUDA_LIB)
    srcs = sorted(os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith(".c"))
    out = os.path.join(LIB, HOST_LIB)
    heads = [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    if not _stale(out, srcs + heads + [cuda_lib, __file__]):
        return out
    cmd = [CC, "-std=gnu11", "-O2", "-fPIC", "-shared", "-Wall", "-Wno-unused-function",
           "-o", out] + srcs + ["-L" + LIB, "-lb200shm", "-Wl,-rpath,$ORIGIN", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("host library build failed:\n" + r.stdout + r.stderr)
    return out


if __name__ == "__main__":
    if "--clean" in sys.argv:
        subprocess.run(["rm", "-rf", OBJ, LIB])
    print(build(verbose=True))
