"""Parity of b200shm_reduce (the sm_100a kernels, through the C ABI) with the
oracle.  Bit-exact everywhere the reference is deterministic; the one
exception, binomial float SUM/PROD, is arrival-order dependent in the
reference and is held to the lowest-mask-first order of the restatement
(bit-exact) and to P*eps*sum|x| of an FP64 sum."""
import zlib

import numpy as np
import pytest

import gen
import oracle

pytestmark = pytest.mark.gpu

NAME = {np.dtype(v): k for k, v in oracle.NP.items()}


def nan_equal_bytes(a, b):
    """Bit equality, except that NaN equals NaN (x86 propagates NaN payloads
    through + and *, the GPU returns the canonical NaN)."""
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    if a.tobytes() == b.tobytes():
        return True
    if a.dtype.kind not in "fc":
        return False
    fa, fb = (a.view(a.real.dtype) if a.dtype.kind == "c" else a), (b.view(b.real.dtype) if b.dtype.kind == "c" else b)
    both_nan = np.isnan(fa) & np.isnan(fb)
    ia = fa.view(np.uint32 if fa.itemsize == 4 else np.uint64)
    ib = fb.view(np.uint32 if fb.itemsize == 4 else np.uint64)
    return bool(((ia == ib) | both_nan).all())


def gpu_reduce(B, heap, algo, op, x, team=None, in_place=False, misalign=0):
    P, N = x.shape
    nb = x[0].nbytes
    team = team or (0, 1, P)
    src = heap(nb + 64) + misalign
    dst = src if in_place else heap(nb + 64) + misalign
    if nb:
        B.put_rows(src, x, team=team)
        if not in_place:
            B.memset(dst, 0xA5, nb, team=team)
    B.reduce(op, NAME[x.dtype], algo, dst, src, N, team=team)
    if not nb:
        return np.zeros_like(x)
    return B.get_rows(dst, nb, x.dtype, team=team)


def combos():
    out = []
    for op in oracle.OPS:
        for dt in ["int8", "int16", "int32", "int64", "uint8", "uint16", "uint32", "uint64",
                   "float32", "float64", "complex64", "complex128"]:
            is_int = dt.startswith(("int", "uint"))
            if op in ("and", "or", "xor") and not is_int:
                continue
            if op in ("min", "max") and dt.startswith("complex"):
                continue
            out.append((op, dt))
    return out


@pytest.mark.parametrize("algo", oracle.ALGOS)
@pytest.mark.parametrize("op,dt", combos())
def test_reduce_matches_oracle(B, heap, rs, algo, op, dt):
    seed = zlib.crc32(f"{algo}{op}{dt}".encode()) & 0xFFFF
    for P, N in [(1, 9), (2, 17), (3, 40), (5, 1), (8, 1000), (13, 77), (32, 131), (64, 257),
                 (100, 45), (128, 37)]:
        x = gen.random_values(oracle.NP[dt], P, N, seed + P)
        if op == "prod" and dt.startswith("float"):
            x = (1.0 + 0.01 * x).astype(x.dtype)
        got = gpu_reduce(B, heap, algo, op, x)
        want = rs.reduce(algo, op, x)
        assert nan_equal_bytes(got, want), (algo, op, dt, P, N)


@pytest.mark.parametrize("algo", oracle.ALGOS)
def test_reduce_zero_elements(B, heap, algo):
    x = np.zeros((4, 0), np.float32)
    gpu_reduce(B, heap, algo, "sum", x)


@pytest.mark.parametrize("algo", ["rec_dbl", "rabenseifner", "binomial", "linear"])
def test_reduce_strided_teams_in_place_and_misaligned(B, heap, rs, algo):
    for team, N in [((3, 2, 5), 129), ((10, 7, 9), 64), ((0, 32, 8), 31), ((255, 1, 1), 5)]:
        P = team[2]
        for dt, op in [("float32", "sum"), ("float64", "prod"), ("int32", "max"), ("uint16", "sum")]:
            x = gen.random_values(oracle.NP[dt], P, N, 7 + P)
            if op == "prod":
                x = (1.0 + 0.01 * x).astype(x.dtype)
            want = rs.reduce(algo, op, x)
            assert nan_equal_bytes(gpu_reduce(B, heap, algo, op, x, team=team), want)
            assert nan_equal_bytes(gpu_reduce(B, heap, algo, op, x, team=team, in_place=True), want)
            mis = 4 if np.dtype(x.dtype).itemsize >= 4 else 2
            assert nan_equal_bytes(gpu_reduce(B, heap, algo, op, x, team=team, misalign=mis), want)


def special(dt, P, N, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((P, N)).astype(dt)
    pick = rng.integers(0, 5, size=(P, N))
    x[pick == 0] = 0.0
    x[pick == 1] = -0.0
    m = rng.random((P, N)) < 0.1
    x[m] = np.nan
    bits = x.view(np.uint32 if np.dtype(dt).itemsize == 4 else np.uint64)
    bits[m] |= rng.integers(1, 1 << 20, size=m.sum()).astype(bits.dtype)
    return x


@pytest.mark.parametrize("algo", oracle.ALGOS)
@pytest.mark.parametrize("dt", ["float32", "float64"])
@pytest.mark.parametrize("op", ["min", "max"])
def test_order_dependent_minmax_is_exact(B, heap, rs, algo, dt, op):
    """NaN payloads and mixed-sign zeros: MIN/MAX select operands, so every
    bit (including which NaN, which zero, and which member gets which under
    rec_dbl) must match the reference's operand order."""
    for P, N, in_place in [(6, 301, False), (8, 64, True), (5, 33, False), (64, 40, True)]:
        x = special(oracle.NP[dt], P, N, P * 31 + N)
        got = gpu_reduce(B, heap, algo, op, x, in_place=in_place)
        assert got.tobytes() == rs.reduce(algo, op, x).tobytes(), (algo, dt, op, P, N, in_place)


@pytest.mark.parametrize("ordered", [False, True])
@pytest.mark.parametrize("dt", ["float32", "float64"])
def test_deferred_list_starts_empty_every_call(B, heap, rs, dt, ordered):
    """The replay kernel of a float MIN/MAX call clears the deferred count
    for the next call (no memset precedes a call).  A call that defers
    nearly every one of 20000 elements is followed by a 100-element call on
    other buffers: a stale count would replay indices far past its rows and
    overwrite the guard bytes after them.  Then a small special-value call.
    `ordered`: the three calls back to back on the engine stream."""
    P = 16
    x1 = special(oracle.NP[dt], P, 20000, 7)
    x2 = gen.normal(oracle.NP[dt], P, 100, 8)
    x3 = special(oracle.NP[dt], P, 37, 9)
    guard = 4096
    bufs = []
    for x in (x1, x2, x3):
        nb = x[0].nbytes
        src, dst = heap(nb), heap(nb + guard)
        B.put_rows(src, x, team=(0, 1, P))
        B.memset(dst, 0xA5, nb + guard, team=(0, 1, P))
        bufs.append((src, dst, nb))
    stream = B.stream() if ordered else None
    for (src, dst, nb), x in zip(bufs, (x1, x2, x3)):
        B.reduce("max", dt, "rec_dbl", dst, src, x.shape[1], team=(0, 1, P), stream=stream)
    if ordered:
        B.quiet()
    for (src, dst, nb), x in zip(bufs, (x1, x2, x3)):
        got = B.get_rows(dst, nb + guard, np.uint8, team=(0, 1, P))
        want = rs.reduce("rec_dbl", "max", x)
        assert got[:, :nb].tobytes() == want.view(np.uint8).tobytes(), (dt, x.shape)
        assert (got[:, nb:] == 0xA5).all(), "bytes after the dest rows were written"


@pytest.mark.parametrize("mis", [8, 4, 1])
def test_sixteen_byte_elements_at_any_alignment(B, heap, rs, mis):
    """complex double (8-byte aligned in C) and long double rows at byte
    offsets that are not multiples of 16: each element moves in 8-, 4- or
    1-byte pieces there, with the same result bits."""
    for algo in ("rec_dbl", "linear"):
        for dt, op in (("complex128", "sum"), ("complex128", "prod"), ("float80", "sum"),
                       ("float80", "max")):
            x = gen.random_values(oracle.NP[dt], 6, 37, 17 + mis)
            if op == "prod":
                x = (1.0 + 0.01 * x).astype(x.dtype)
            got = gpu_reduce(B, heap, algo, op, x, misalign=mis)
            want = rs.reduce(algo, op, x)
            if dt == "float80":
                vb = lambda a: np.ascontiguousarray(a).view(np.uint8).reshape(a.shape + (16,))[..., :10]
                assert vb(got).tobytes() == vb(want).tobytes(), (algo, dt, op, mis)
            else:
                assert nan_equal_bytes(got, want), (algo, dt, op, mis)


@pytest.mark.parametrize("dt", ["complex64", "complex128"])
def test_complex_prod_with_infinities(B, heap, rs, dt):
    rng = np.random.default_rng(5)
    x = (rng.standard_normal((4, 64)) + 1j * rng.standard_normal((4, 64))).astype(dt)
    x[0, :8] = complex(np.inf, 1.0)
    x[1, 4:12] = complex(np.nan, np.inf)
    x[2, 20:24] = complex(0.0, np.nan)
    for algo in ("rec_dbl", "linear"):
        got = gpu_reduce(B, heap, algo, "prod", x)
        want = rs.reduce(algo, "prod", x)
        assert nan_equal_bytes(got, want), algo


def test_binomial_float_within_fp64_bound(B, heap):
    x = gen.normal(np.float32, 13, 4096, 99)
    got = gpu_reduce(B, heap, "binomial", "sum", x)
    exact = x.astype(np.float64).sum(0)
    bound = 13 * np.finfo(np.float32).eps * np.abs(x.astype(np.float64)).sum(0)
    assert (np.abs(got.astype(np.float64) - exact) <= bound).all()


@pytest.mark.parametrize("algo", ["rec_dbl", "rabenseifner"])
def test_config2_full_size(B, rs, algo):
    """Config 2 at full size: 64 PEs x 2^20 elements, f32 SUM (N(0,1)),
    f64 MAX (uniform +-1e6), i64 XOR (uniform bits); bit-exact against the
    restatement, and f32 within P*eps*sum|x| of an FP64 sum."""
    import b200shm
    P, N = 64, 1 << 20
    off_s = b200shm.malloc(8 * N)
    off_d = b200shm.malloc(8 * N)
    try:
        for dt, op, x in [("float32", "sum", gen.normal(np.float32, P, N, 21)),
                          ("float64", "max", gen.uniform(np.float64, P, N, 22, -1e6, 1e6)),
                          ("int64", "xor", gen.uniform_int(np.int64, P, N, 23))]:
            team = (0, 1, P)
            b200shm.put_rows(off_s, x, team=team)
            b200shm.reduce(op, dt, algo, off_d, off_s, N, team=team)
            got = b200shm.get_rows(off_d, x[0].nbytes, x.dtype, team=team)
            want = rs.reduce(algo, op, x)
            assert got.tobytes() == want.tobytes(), (dt, op)
            if dt == "float32":
                exact = x.astype(np.float64).sum(0)
                err = np.abs(got[0].astype(np.float64) - exact).max()
                scale = np.abs(x.astype(np.float64)).sum(0)
                assert (np.abs(got[0] - exact) <= P * np.finfo(np.float32).eps * scale).all(), err
    finally:
        b200shm.free(off_s)
        b200shm.free(off_d)


def test_reduce_rejects_bad_arguments(B, heap):
    src = heap(4096)
    with pytest.raises(B.B200Error):
        B.reduce("xor", "float32", "rec_dbl", src, src, 16, team=(0, 1, 4))
    with pytest.raises(B.B200Error):
        B.reduce("xor", "float80", "rec_dbl", src, src, 16, team=(0, 1, 4))
    with pytest.raises(B.B200Error):
        B.reduce("sum", "float32", "rec_dbl", src + 8, src, 16, team=(0, 1, 4))  # partial overlap
    with pytest.raises(B.B200Error):
        B.reduce("sum", "float32", "rec_dbl", src, src, 16, team=(250, 1, 16))  # past npes
    with pytest.raises(B.B200Error):
        B.reduce("sum", "int32", "rec_dbl", src, src, 1 << 40, team=(0, 1, 4))  # past slice
