"""Long double reductions (shmem_longdouble_<op>_reduce) on the GPU, through
the C ABI, against the oracle run on this host's x87 unit: the 10 bytes
that carry each value bit for bit (6 bytes of every 16 are padding), for
every algorithm and MIN/MAX/SUM/PROD, on values with full 64-bit
significands, and on operands of every encoding class (zeros of both
signs, infinities, quiet and signalling NaNs with payloads, denormals,
pseudo-denormals and unnormals), where MIN/MAX under rec_dbl gives
different members different bits, as the reference does."""
import platform

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

if platform.machine() not in ("x86_64", "AMD64") or np.dtype(np.longdouble).itemsize != 16:
    pytest.skip("needs the x86-64 long double", allow_module_level=True)

BIAS = 16383


def pack(se, sig):
    """long double array from sign+exponent (uint16) and significand (uint64)."""
    se = np.asarray(se, np.uint16)
    sig = np.asarray(sig, np.uint64)
    raw = np.zeros(se.shape + (16,), np.uint8)
    raw[..., :8] = sig[..., None].view(np.uint8).reshape(sig.shape + (8,))
    raw[..., 8:10] = se[..., None].view(np.uint8).reshape(se.shape + (2,))
    return raw.view(np.longdouble).reshape(se.shape)


def value_bytes(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint8).reshape(a.shape + (16,))[..., :10].tobytes()


def full_precision(P, N, seed, spread):
    """Normal values with random 64-bit significands, exponents within
    `spread` of 1.0, random signs."""
    rng = np.random.default_rng(seed)
    sig = rng.integers(0, 2 ** 63, size=(P, N), dtype=np.uint64) | np.uint64(1 << 63)
    e = BIAS + rng.integers(-spread, spread + 1, size=(P, N))
    s = rng.integers(0, 2, size=(P, N)) << 15
    return pack(e | s, sig)


def specials(P, N, seed):
    """A mix of every encoding class (about 1/3 of the values special)."""
    rng = np.random.default_rng(seed)
    x = full_precision(P, N, seed, 8)
    se = x.view(np.uint8).reshape(P, N, 16)[..., 8:10].copy().view(np.uint16)[..., 0]
    sig = x.view(np.uint8).reshape(P, N, 16)[..., :8].copy().view(np.uint64)[..., 0]
    pick = rng.integers(0, 27, size=(P, N))
    s = (rng.integers(0, 2, size=(P, N)) << 15).astype(np.uint16)
    pay = rng.integers(1, 1 << 20, size=(P, N)).astype(np.uint64)
    J, Q = np.uint64(1 << 63), np.uint64(1 << 62)
    table = {
        0: (s, np.uint64(0)),                                       # +-0
        1: (s, np.uint64(0)),
        2: (s | 0x7FFF, J),                                         # +-inf
        3: (s | 0x7FFF, J | Q | pay),                               # quiet NaN
        4: (s | 0x7FFF, J | pay),                                   # signalling NaN
        5: (s, pay),                                                # denormal
        6: (s, J | pay),                                            # pseudo-denormal
        7: (s | np.uint16(BIAS), pay),                              # unnormal
        8: (s | np.uint16(1), J | pay),                             # smallest normals
    }
    for k, (e_k, m_k) in table.items():
        m = pick == k
        se[m] = np.broadcast_to(e_k, (P, N))[m]
        sig[m] = np.broadcast_to(m_k, (P, N))[m]
    return pack(se, sig)


def run(B, heap, algo, op, x, in_place=False):
    P, N = x.shape
    nb = x[0].nbytes
    src = heap(nb)
    dst = src if in_place else heap(nb)
    B.put_rows(src, x, team=(0, 1, P))
    B.reduce(op, "float80", algo, dst, src, N, team=(0, 1, P))
    return B.get_rows(dst, nb, np.longdouble, team=(0, 1, P))


@pytest.mark.parametrize("algo", oracle.ALGOS)
@pytest.mark.parametrize("op", ["min", "max", "sum", "prod"])
def test_longdouble_reduce_full_precision(B, heap, rs, algo, op):
    for P, N, spread in [(5, 33, 40), (8, 257, 3), (64, 100, 1), (100, 19, 2)]:
        x = full_precision(P, N, P * 7 + N, spread)
        got = run(B, heap, algo, op, x)
        assert value_bytes(got) == value_bytes(rs.reduce(algo, op, x)), (algo, op, P, N)


@pytest.mark.parametrize("algo", oracle.ALGOS)
@pytest.mark.parametrize("op", ["min", "max", "sum", "prod"])
def test_longdouble_reduce_every_encoding(B, heap, rs, algo, op):
    for P, N, in_place in [(6, 301, False), (8, 64, True), (33, 40, False)]:
        x = specials(P, N, P * 131 + N)
        got = run(B, heap, algo, op, x, in_place=in_place)
        assert value_bytes(got) == value_bytes(rs.reduce(algo, op, x)), (algo, op, P, N)


def test_longdouble_against_the_reference_build(B, heap, ref):
    """The same comparison with the reference's own code (oracle/_ref)."""
    for op in ["min", "max", "sum", "prod"]:
        for algo in ["rec_dbl", "rabenseifner", "linear"]:
            x = specials(8, 64, 99) if op in ("min", "max") else full_precision(8, 64, 98, 2)
            want, _ = ref.reduce(algo, op, x)
            got = run(B, heap, algo, op, x)
            assert value_bytes(got) == value_bytes(want), (algo, op)


def test_longdouble_through_the_noalloc_entry(B, heap, rs):
    """b200shm_reduce_noalloc on the heap's own rows gives the same bits."""
    import ctypes
    x = specials(8, 500, 5)
    P, N = x.shape
    nb = x[0].nbytes
    src, dst = heap(nb), heap(nb)
    B.put_rows(src, x, team=(0, 1, P))
    L = B.lib
    L.b200shm_reduce_noalloc.argtypes = [ctypes.c_int] * 4 + [
        ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
        ctypes.c_void_p]
    slice_ = L.b200shm_heap_slice()
    base = L.b200shm_heap_base()
    rc = L.b200shm_reduce_noalloc(B.OPS.index("max"), B.DTYPES.index("float80"),
                                  B.ALGOS.index("rec_dbl"), P, base + dst, slice_, base + src,
                                  slice_, N, None)
    assert rc == 0, L.b200shm_last_error()
    got = B.get_rows(dst, nb, np.longdouble, team=(0, 1, P))
    assert value_bytes(got) == value_bytes(rs.reduce("rec_dbl", "max", x))
