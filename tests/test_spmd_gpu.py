"""The OpenSHMEM surface (include/shmem.h over libshmem_b200.so): a C program
written like any OpenSHMEM program (tests/c/spmd_parity.c, 8 PEs) must leave
in every PE exactly what the reference's algorithms leave there."""
import os
import subprocess

import numpy as np
import pytest

import gen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "osss-ucx_b200", "lib")
NP, NR, NFC, NFS, NDM, BLK, NAS = 8, 1024, 256, 4096, 512, 96, 5

OUT = np.dtype([("red", np.int32, (NP, NR)), ("fc", np.int64, (NP, NP * NFC)),
                ("fs", np.float32, (NP, NFS)), ("dm", np.float64, (NP, NDM)),
                ("toall", np.int32, (NP, NR)), ("team_even", np.int32, (NP, NR)),
                ("a2a", np.uint8, (NP, NP * BLK)), ("as", np.int64, (NP, NP * NAS * 2)),
                ("bcast", np.int64, (NP, NFC)), ("amo_final", np.int64),
                ("amo_fetched", np.int64, (NP, 4)), ("team_info", np.int32, (NP, 4)),
                ("status", np.int32, (NP,))], align=True)


def compile_program(tmp_path):
    import __graft_entry__
    __graft_entry__.build_library()
    exe = str(tmp_path / "spmd_parity")
    subprocess.run(["gcc", "-std=gnu11", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "spmd_parity.c"), "-L" + LIB,
                    "-lshmem_b200", "-Wl,-rpath," + LIB, "-o", exe], check=True)
    return exe


def test_program_compiles_and_links_against_the_surface(tmp_path):
    assert os.path.exists(compile_program(tmp_path))


def special_doubles(P, N, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1e6, 1e6, (P, N))
    pick = rng.integers(0, 8, size=(P, N))
    x[pick == 0] = 0.0
    x[pick == 1] = -0.0
    x[pick == 2] = np.nan
    return x


@pytest.mark.gpu
def test_spmd_program_matches_oracle(tmp_path, rs):
    exe = compile_program(tmp_path)
    red, fc = gen.config1_inputs()
    fs = gen.normal(np.float32, NP, NFS, 5)
    dm = special_doubles(NP, NDM, 6)
    a2a = gen.uniform_int(np.uint8, NP, NP * BLK, 7)
    as_ = gen.uniform_int(np.int64, NP, NP * NAS * 3, 8)
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        for a in (red, fc, fs, dm, a2a, as_):
            f.write(np.ascontiguousarray(a).tobytes())
    outp = tmp_path / "out.bin"
    env = dict(os.environ, SHMEM_SYMMETRIC_SIZE="16M")
    r = subprocess.run([exe, str(inp), str(outp)], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    o = np.fromfile(outp, dtype=OUT)[0]
    assert (o["status"] == 0).all()
    assert o["red"].tobytes() == rs.reduce("rec_dbl", "sum", red).tobytes()
    assert o["fc"].tobytes() == rs.fcollect(fc).tobytes()
    assert o["fs"].tobytes() == rs.reduce("rec_dbl", "sum", fs).tobytes()
    assert o["dm"].tobytes() == rs.reduce("rec_dbl", "max", dm).tobytes()
    assert o["toall"].tobytes() == o["red"].tobytes()
    even = rs.reduce("rec_dbl", "sum", red[0::2])
    assert o["team_even"][0::2].tobytes() == even.tobytes()
    assert (o["team_even"][1::2] == 0).all()
    assert o["a2a"].tobytes() == rs.alltoall(a2a).tobytes()
    assert o["as"].tobytes() == rs.alltoalls(as_, np.zeros((NP, NP * NAS * 2), np.int64), 2, 3,
                                             NAS).tobytes()
    want_b = np.zeros((NP, NFC), np.int64)
    assert o["bcast"].tobytes() == rs.broadcast(fc, want_b, 3).tobytes()
    assert o["amo_final"] == NP * 4
    assert sorted(o["amo_fetched"].ravel().tolist()) == list(range(NP * 4))
    assert all(list(row) == sorted(row) for row in o["amo_fetched"].tolist())
    info = o["team_info"]
    for pe in range(NP):
        if pe % 2 == 0:
            assert info[pe][0] == pe // 2 and info[pe][1] == NP // 2
        else:
            assert info[pe][0] == -1 and info[pe][1] == -1
        assert info[pe][2] == (pe % 4) * 100 + 4
        assert info[pe][3] == (pe // 4) * 100 + 2


NC = 6
OUTC = np.dtype([("c32", np.int32, (NC, 3 * NC * (NC + 1) // 2)), ("c64", np.int64, (NC, 15)),
                 ("cm", np.uint8, (NC, 5 * NC + NC * (NC - 1) // 2)), ("status", np.int32, (NC,))],
                align=True)


@pytest.mark.gpu
def test_spmd_collect_matches_oracle(tmp_path, rs):
    """shmem_int32_collect (team), shmem_collect64 (active set of the even
    PEs) and shmem_collectmem, each PE passing its own count."""
    import __graft_entry__
    __graft_entry__.build_library()
    exe = str(tmp_path / "spmd_collect")
    subprocess.run(["gcc", "-std=gnu11", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "spmd_collect.c"), "-L" + LIB,
                    "-lshmem_b200", "-Wl,-rpath," + LIB, "-o", exe], check=True)
    outp = tmp_path / "out.bin"
    r = subprocess.run([exe, str(outp)], env=dict(os.environ, SHMEM_SYMMETRIC_SIZE="8M"),
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    o = np.fromfile(outp, dtype=OUTC)[0]
    assert (o["status"] == 0).all()
    c32 = [3 * (i + 1) for i in range(NC)]
    x = np.zeros((NC, max(c32)), np.int32)
    for i in range(NC):
        x[i, :c32[i]] = i * 1000 + np.arange(c32[i])
    want = rs.collect(x.view(np.uint8), [c * 4 for c in c32], sum(c32) * 4)
    assert o["c32"].tobytes() == want.tobytes()
    evens = [0, 2, 4]
    c64 = [2 * i + 1 for i in evens]
    x = np.zeros((3, max(c64)), np.int64)
    for k, i in enumerate(evens):
        x[k, :c64[k]] = (i << 40) | np.arange(c64[k])
    want = rs.collect(x.view(np.uint8), [c * 8 for c in c64], sum(c64) * 8)
    assert o["c64"][evens].tobytes() == want.tobytes()
    assert (o["c64"][1::2] == 0).all()
    cm = [5 + i for i in range(NC)]
    x = np.zeros((NC, max(cm)), np.uint8)
    for i in range(NC):
        x[i, :cm[i]] = (i * 16 + np.arange(cm[i])) & 0xFF
    assert o["cm"].tobytes() == rs.collect(x, cm, sum(cm)).tobytes()


NN, NB, NADD = 8, 64, 16
OUTN = np.dtype([("dst", np.int64, (NN, NN * NB)), ("got", np.int64, (NN, NB)),
                 ("fetched", np.int64, (NN, NADD)), ("loc", np.uint8, (NN, NN * 32)),
                 ("counter", np.int64), ("status", np.int32, (NN,))], align=True)


@pytest.mark.gpu
def test_spmd_nbi_through_the_serving_loop(tmp_path):
    """shmem_int64_put_nbi / get_nbi, shmem_int64_atomic_fetch_add_nbi and
    shmem_quiet: puts land in the next PE, gets bring the previous PE's
    block, the counter adds up and hands out every value exactly once."""
    import __graft_entry__
    __graft_entry__.build_library()
    exe = str(tmp_path / "spmd_nbi")
    subprocess.run(["gcc", "-std=gnu11", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "spmd_nbi.c"), "-L" + LIB,
                    "-lshmem_b200", "-Wl,-rpath," + LIB, "-o", exe], check=True)
    outp = tmp_path / "out.bin"
    r = subprocess.run([exe, str(outp)], env=dict(os.environ, SHMEM_SYMMETRIC_SIZE="8M"),
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    o = np.fromfile(outp, dtype=OUTN)[0]
    assert (o["status"] == 0).all()
    src = np.array([[p * 1000 + i for i in range(NB)] for p in range(NN)], np.int64)
    for p in range(NN):
        want = np.zeros(NN * NB, np.int64)
        q = (p - 1) % NN
        want[q * NB:(q + 1) * NB] = src[q]
        assert (o["dst"][p] == want).all()
        assert (o["got"][p] == src[(p - 1) % NN]).all()
    assert o["counter"] == NN * NADD
    assert sorted(o["fetched"].ravel().tolist()) == list(range(NN * NADD))
    want_loc = np.zeros(NN * 32, np.uint8)
    for p in range(NN):
        want_loc[p * 32:(p + 1) * 32] = (p * 32 + np.arange(32)) & 0xFF
    assert (o["loc"][0] == want_loc).all()


TP = 4
OUTX = np.dtype([("dst", np.int64, (NN, NN * NB)), ("tdst", np.int64, (NN, TP * NB)),
                 ("fa", np.int64, (NN, NADD)), ("fc", np.int64, (NN,)), ("g", np.int64, (NN,)),
                 ("counter", np.int64), ("counter2", np.int64), ("bits", np.int64),
                 ("pending", np.int32, (NN, 6)), ("create_rc", np.int32, (NN,)),
                 ("team_rc", np.int32, (NN,)), ("team_ok", np.int32, (NN,)),
                 ("invalid_status", np.int32, (NN,)), ("status", np.int32, (NN,))], align=True)


@pytest.mark.gpu
def test_spmd_contexts_quiet_independently(tmp_path):
    """shmem_ctx_create / quiet / destroy, shmem_team_create_ctx: quieting one
    context completes its operations and leaves another's pending; a team
    context takes team-relative PE numbers; destroying a context completes
    it; SHMEM_CTX_INVALID is refused."""
    import __graft_entry__
    __graft_entry__.build_library()
    exe = str(tmp_path / "spmd_ctx")
    subprocess.run(["gcc", "-std=gnu11", "-O2", "-Wall", "-Werror",
                    "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "spmd_ctx.c"), "-L" + LIB,
                    "-lshmem_b200", "-Wl,-rpath," + LIB, "-o", exe], check=True)
    outp = tmp_path / "out.bin"
    r = subprocess.run([exe, str(outp)], env=dict(os.environ, SHMEM_SYMMETRIC_SIZE="8M"),
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert os.path.getsize(outp) == OUTX.itemsize
    o = np.fromfile(outp, dtype=OUTX)[0]
    assert (o["status"] == 0).all() and (o["create_rc"] == 0).all()
    assert (o["pending"] == [NADD, 1, 0, 1, 0, 0]).all(), o["pending"]
    assert o["counter"] == NN * NADD
    assert sorted(o["fa"].ravel().tolist()) == list(range(NN * NADD))
    src = np.array([[p * 1000 + i for i in range(NB)] for p in range(NN)], np.int64)
    for p in range(NN):
        want = np.zeros(NN * NB, np.int64)
        q = (p - 1) % NN
        want[q * NB:(q + 1) * NB] = src[q]
        assert (o["dst"][p] == want).all()
    even = list(range(0, NN, 2))
    assert [int(v == 0) for v in o["team_rc"]] == [int(p in even) for p in range(NN)]
    assert (o["team_ok"] == 1).all()
    for p in even:
        want = np.zeros(TP * NB, np.int64)
        tq = (p // 2 - 1) % TP
        want[tq * NB:(tq + 1) * NB] = src[2 * tq]
        assert (o["tdst"][p] == want).all()
    for p in range(1, NN, 2):
        assert (o["tdst"][p] == 0).all()
    assert o["bits"] == sum(1 << p for p in even)
    assert o["counter2"] == NN and sorted(o["fc"].tolist()) == list(range(NN))
    assert (o["invalid_status"] < 0).all()
    assert (o["g"] == np.arange(NN)).all()


@pytest.mark.gpu
def test_spmd_point_to_point_sync_and_signalled_puts(tmp_path):
    """tests/c/spmd_sync.c checks itself: strided iput/iget (typed and
    sized), put_signal with signal_wait_until / signal_fetch, the
    test/wait_until families with status masks and vector compare values,
    unsigned comparison, and that a collective whose members disagree fails
    on every member with the same message."""
    import __graft_entry__
    __graft_entry__.build_library()
    exe = str(tmp_path / "spmd_sync")
    subprocess.run(["gcc", "-std=gnu11", "-O2", "-Wall", "-Werror",
                    "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "spmd_sync.c"), "-L" + LIB,
                    "-lshmem_b200", "-Wl,-rpath," + LIB, "-o", exe], check=True)
    r = subprocess.run([exe], env=dict(os.environ, SHMEM_SYMMETRIC_SIZE="8M",
                                       SHMEM_B200_WAIT_TIMEOUT="60"),
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr


def compile_generics(tmp_path):
    import __graft_entry__
    __graft_entry__.build_library()
    exe = str(tmp_path / "spmd_generics")
    subprocess.run(["gcc", "-std=c11", "-O2", "-Wall", "-Wextra", "-Werror",
                    "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "spmd_generics.c"), "-L" + LIB,
                    "-lshmem_b200", "-Wl,-rpath," + LIB, "-o", exe], check=True)
    return exe


def test_generic_names_resolve_to_the_typed_functions(tmp_path):
    """The C11 generic names compile (C11, every warning an error) and link
    in a program that uses them on a dozen types, with and without a
    context first; the sized typedefs select the functions of the types
    they alias; a generic call on a type outside its table does not
    compile."""
    assert os.path.exists(compile_generics(tmp_path))
    inc = "-I" + os.path.join(ROOT, "include")
    good = tmp_path / "good.c"
    good.write_text(
        '#include <stdint.h>\n#include "shmem.h"\n'
        "int64_t f(int64_t *c, uint32_t *u, size_t *s, int8_t *d, const int8_t *x) {\n"
        "  shmem_atomic_fetch_and(u, 3u, 0);\n"
        "  shmem_atomic_add(s, (size_t)1, 0);\n"
        "  shmem_and_reduce(SHMEM_TEAM_WORLD, d, x, 4);\n"
        "  return shmem_atomic_fetch_add(c, (int64_t)1, 0);\n}\n")
    r = subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-fsyntax-only", inc, str(good)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    bad = tmp_path / "bad.c"
    bad.write_text('#include "shmem.h"\n'
                   "float f(float *p) { return shmem_atomic_fetch_add(p, 1.0f, 0); }\n")
    r = subprocess.run(["gcc", "-std=c11", "-fsyntax-only", inc, str(bad)],
                       capture_output=True, text=True)
    assert r.returncode != 0 and "b200_shmem_generic_type_error" in r.stderr, r.stderr


@pytest.mark.gpu
def test_spmd_generics_program(tmp_path):
    """tests/c/spmd_generics.c checks itself: generic RMA, atomics (and the
    pre-1.4 names), reductions, collectives and waits; locks around a
    read-modify-write; realloc; the version, name and state queries."""
    exe = compile_generics(tmp_path)
    r = subprocess.run([exe], env=dict(os.environ, SHMEM_SYMMETRIC_SIZE="8M",
                                       SHMEM_B200_WAIT_TIMEOUT="60"),
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr


@pytest.mark.gpu
def test_spmd_longdouble_reductions(tmp_path, rs):
    """shmem_longdouble_sum_reduce / _prod_reduce over SHMEM_TEAM_WORLD and
    shmem_longdouble_max_to_all (NaN payloads, signed zeros, infinities
    among the inputs) from an 8-PE C program, against the oracle on the
    10 value bytes of every element (tests/c/spmd_longdouble.c)."""
    import __graft_entry__
    __graft_entry__.build_library()
    exe = str(tmp_path / "spmd_longdouble")
    subprocess.run(["gcc", "-std=gnu11", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "spmd_longdouble.c"), "-L" + LIB,
                    "-lshmem_b200", "-Wl,-rpath," + LIB, "-o", exe], check=True)
    P, N = 8, 300
    rng = np.random.default_rng(11)
    s = (1.0 + rng.uniform(-0.25, 0.25, (P, N))).astype(np.longdouble)
    s *= (1.0 + np.longdouble(2.0) ** -40 * rng.integers(0, 1 << 20, (P, N)))  # full significands
    m = rng.uniform(-1e6, 1e6, (P, N)).astype(np.longdouble)
    pick = rng.integers(0, 8, size=(P, N))
    m[pick == 0] = 0.0
    m[pick == 1] = -0.0
    m[pick == 2] = np.nan
    m[pick == 3] = -np.inf
    inp, outp = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(inp, "wb") as f:
        f.write(np.ascontiguousarray(s).tobytes())
        f.write(np.ascontiguousarray(m).tobytes())
    r = subprocess.run([exe, str(inp), str(outp)], env=dict(os.environ, SHMEM_SYMMETRIC_SIZE="8M"),
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    raw = np.fromfile(outp, dtype=np.uint8)
    n = P * N * 16
    got = [raw[i * n:(i + 1) * n].view(np.longdouble).reshape(P, N) for i in range(3)]
    assert (raw[3 * n:].view(np.int32) == 0).all()

    def vb(a):
        return np.ascontiguousarray(a).view(np.uint8).reshape(P, N, 16)[..., :10].tobytes()
    assert vb(got[0]) == vb(rs.reduce("rec_dbl", "sum", s))
    assert vb(got[1]) == vb(rs.reduce("rec_dbl", "prod", s))
    assert vb(got[2]) == vb(rs.reduce("rec_dbl", "max", m))
