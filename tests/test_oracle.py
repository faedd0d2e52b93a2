"""The CPU restatement is pinned against the reference's own code.

* every golden fixture (outputs of the reference's src/shcoll/src code over
  emulated PEs, tests/golden/make_golden.py) is reproduced bit for bit;
* where the reference tree is present (oracle/_ref), random sweeps over
  types x ops x algorithms x team sizes compare the two directly.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import gen
import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SHMEM_T = {"int8": "int8", "int16": "int16", "int32": "int32", "int64": "int64",
           "uint8": "uint8", "uint16": "uint16", "uint32": "uint32", "uint64": "uint64",
           "float32": "float", "float64": "double", "float80": "longdouble",
           "complex64": "complexf", "complex128": "complexd"}


def value_bytes(a):
    """Bytes that carry the value (long double has 6 padding bytes)."""
    a = np.ascontiguousarray(a)
    if a.dtype == np.longdouble:
        return a.view(np.uint8).reshape(a.shape + (16,))[..., :10].tobytes()
    return a.tobytes()


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def test_manifest_matches_fixtures():
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        manifest = json.load(f)
    for fname, digests in manifest.items():
        z = load(fname)
        assert sorted(z.files) == sorted(digests)
        for k, d in digests.items():
            assert hashlib.sha256(np.ascontiguousarray(z[k]).tobytes()).hexdigest() == d


def test_golden_config1(rs):
    z = load("config1.npz")
    x, fc = gen.config1_inputs()
    assert np.array_equal(z["reduce_in"], x) and np.array_equal(z["fcollect_in"], fc)
    assert rs.reduce("rec_dbl", "sum", x).tobytes() == z["reduce_out"].tobytes()
    assert rs.fcollect(fc).tobytes() == z["fcollect_out"].tobytes()
    # the known answer itself: every PE holds the column sums / the PE-ordered concat
    assert np.array_equal(z["reduce_out"], np.broadcast_to(x.sum(0, dtype=np.int32), x.shape))
    assert np.array_equal(z["fcollect_out"], np.broadcast_to(fc.reshape(-1), (8, 8 * 256)))


def golden_reduce_cases():
    z = load("reduce.npz")
    names = sorted({k.rsplit("/", 1)[0] for k in z.files})
    return [(n, z[n + "/in"], z[n + "/out"]) for n in names]


@pytest.mark.parametrize("case", golden_reduce_cases(), ids=lambda c: c[0])
def test_golden_reduce(rs, case):
    name, x, y = case
    parts = name.split("/")
    algo, op = (parts[1], parts[2]) if parts[0] == "special" else (parts[0], parts[1])
    assert rs.reduce(algo, op, x).tobytes() == y.tobytes()


def test_golden_copy(rs):
    z = load("copy.npz")
    assert rs.fcollect(z["fcollect/in"]).tobytes() == z["fcollect/out"].tobytes()
    assert rs.alltoall(z["alltoall/in"]).tobytes() == z["alltoall/out"].tobytes()
    got = rs.alltoalls(z["alltoalls/in"], z["alltoalls/dest0"], 2, 3, 5)
    assert got.tobytes() == z["alltoalls/out"].tobytes()


def test_reverse_bits(rs):
    for n in range(0, 12):
        for x in range(1 << n):
            want = int(format(x, "0%db" % n)[::-1], 2) if n else 0
            assert rs.L.or_reverse_bits(x, n) == want


def test_rec_dbl_members_differ_only_when_order_matters(rs):
    """rec_dbl leaves different bits in different members for MIN with
    mixed-sign zeros (each member computes op(own, partner's))."""
    x = np.array([[0.0], [-0.0], [0.0], [-0.0]], dtype=np.float64)
    y = rs.reduce("rec_dbl", "min", x)
    signs = np.signbit(y[:, 0])
    assert signs.any() and not signs.all()
    y2 = rs.reduce("rabenseifner", "min", x)
    assert len({v.tobytes() for v in y2}) == 1


# ---------------------------------------------------------------------------
# direct comparison with the reference build (skipped without oracle/_ref)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("algo", oracle.ALGOS)
def test_restatement_matches_reference_reduce(rs, ref, algo):
    rng = np.random.default_rng(oracle.ALGOS.index(algo))
    for op in oracle.OPS:
        for tname in oracle.reduce_types(op):
            dt = oracle.SHMEM_TYPES[tname]
            if algo == "binomial" and dt.startswith(("float", "complex")):
                continue  # covered by the tolerance test below
            for P in (1, 2, 3, 7, 8):
                N = int(rng.integers(0, 24))
                x = gen.random_values(oracle.NP[dt], P, N, int(rng.integers(1 << 30)))
                got = rs.reduce(algo, op, x)
                want, _ = ref.reduce(algo, op, x, tname=tname)
                assert value_bytes(got) == value_bytes(want), (algo, op, tname, P, N)


def test_reference_to_all_form_matches(rs, ref):
    rng = np.random.default_rng(3)
    for algo in ("rec_dbl", "rabenseifner", "linear"):
        for tname, op in (("int", "sum"), ("double", "sum"), ("long", "xor"), ("float", "max")):
            dt = oracle.SHMEM_TYPES[tname]
            x = gen.random_values(oracle.NP[dt], 6, 19, int(rng.integers(1 << 30)))
            want, _ = ref.reduce(algo, op, x, tname=tname, form="to_all")
            assert rs.reduce(algo, op, x).tobytes() == want.tobytes()


def test_reference_binomial_float_within_tolerance(rs, ref):
    """The reference's binomial reduce folds children in message-arrival
    order (reduce.c:137-154), so its float sums vary from run to run; they
    all stay within P*eps*sum|x| of the exact sum, as does the restatement."""
    x = gen.normal(np.float64, 13, 64, 11)
    exact = x.sum(0)
    bound = 13 * np.finfo(np.float64).eps * np.abs(x).sum(0)
    for _ in range(5):
        y, _ = ref.reduce("binomial", "sum", x, tname="double")
        assert (np.abs(y - exact) <= bound).all()
    assert (np.abs(rs.reduce("binomial", "sum", x) - exact) <= bound).all()


def test_restatement_matches_reference_copies(rs, ref):
    rng = np.random.default_rng(9)
    fc_algos = ["linear", "all_linear", "all_linear1", "rec_dbl", "ring", "bruck",
                "bruck_no_rotate", "bruck_signal", "bruck_inplace", "neighbor_exchange"]
    for algo in fc_algos:
        for P in (1, 2, 4, 6, 8):
            if algo == "rec_dbl" and P & (P - 1):
                continue
            if algo == "neighbor_exchange" and P % 2:
                continue
            x = rng.integers(-2**31, 2**31, size=(P, 9)).astype(np.int64)
            out = np.zeros((P, P * 9), np.int64)
            ref.run(oracle.K_SIZED, f"shcoll_fcollect64_{algo}", x, out, nelems=9)
            assert rs.fcollect(x).tobytes() == out.tobytes(), (algo, P)
    for base in ("shift_exchange", "xor_pairwise_exchange", "color_pairwise_exchange"):
        for sync in ("barrier", "counter", "signal"):
            for P in (1, 2, 4, 6):
                if base.startswith("xor") and P & (P - 1):
                    continue
                if base.startswith("color") and P % 2:
                    continue
                x = rng.integers(0, 2**32, size=(P, P * 5)).astype(np.uint32)
                out = np.zeros_like(x)
                ref.run(oracle.K_SIZED, f"shcoll_alltoall32_{base}_{sync}", x, out, nelems=5)
                assert rs.alltoall(x).tobytes() == out.tobytes(), (base, sync, P)
    for base in ("shift_exchange", "xor_pairwise_exchange", "color_pairwise_exchange"):
        for sync in ("barrier", "counter"):
            for P in (2, 4):
                for dst, sst in ((1, 1), (2, 3), (3, 2)):
                    n = 4
                    x = rng.integers(-2**40, 2**40, size=(P, P * n * sst)).astype(np.int64)
                    d0 = rng.integers(-9, 9, size=(P, P * n * dst)).astype(np.int64)
                    out = d0.copy()
                    ref.run(oracle.K_ALLTOALLS_SIZED, f"shcoll_alltoalls64_{base}_{sync}", x, out,
                            nelems=n, a=dst, b=sst)
                    got = rs.alltoalls(x, d0, dst, sst, n)
                    assert got.tobytes() == out.tobytes(), (base, sync, P, dst, sst)


COLLECT_ALGOS = ["linear", "all_linear", "all_linear1", "rec_dbl", "rec_dbl_signal", "ring",
                 "bruck", "bruck_no_rotate"]


@pytest.mark.parametrize("algo", COLLECT_ALGOS)
def test_restatement_matches_reference_collect(rs, ref, algo):
    """Collect with a different count on every member (member i passes
    base + (i*a) % (b+1), the rule the emulator applies): the reference's
    sized (32/64) and team (typed, mem) forms against the restatement.
    collect_helper_simple is left out: it copies each PE's block into its own
    dest only (collect.c:35-52), so it exchanges no data; so is linear over a
    single PE, which adds to PE me + stride outside the set (collect.c:80)."""
    rng = np.random.default_rng(17)
    sizes = (1, 2, 4, 8) if algo.startswith("rec_dbl") else (1, 2, 3, 5, 8)
    if algo == "linear":
        sizes = sizes[1:]
    for P in sizes:
        for base, a, b in ((3, 5, 6), (0, 2, 3), (11, 1, 1)):
            counts = [base + (i * a) % (b + 1) for i in range(P)]
            for es, tag in ((4, "collect32"), (8, "collect64")):
                x = rng.integers(0, 256, size=(P, max(max(counts) * es, 1)), dtype=np.uint8)
                tot = sum(counts) * es
                out = np.zeros((P, tot + 16), np.uint8)
                ref.run(oracle.K_COLLECT_SIZED, f"shcoll_{tag}_{algo}", x, out, nelems=base, a=a,
                        b=b)
                want = rs.collect(x, [c * es for c in counts], tot + 16)
                assert out.tobytes() == want.tobytes(), (algo, P, base, a, b, es)
            if algo.startswith("rec_dbl"):
                continue
            x = rng.integers(0, 256, size=(P, max(max(counts) * 8, 1)), dtype=np.uint8)
            out = np.zeros((P, sum(counts) * 8 + 8), np.uint8)
            ref.run(oracle.K_COLLECT_TEAM, f"shcoll_int64_collect_{algo}", x, out, nelems=base,
                    a=a, b=b)
            want = rs.collect(x, [c * 8 for c in counts], sum(counts) * 8 + 8)
            assert out.tobytes() == want.tobytes(), (algo, P, "team")


# ---------------------------------------------------------------------------
# the restatement against the reference at the team sizes and shapes the
# GPU is run at (deeper butterflies, extra-PE folds of large teams, the
# configured element counts)
# ---------------------------------------------------------------------------
LARGE_TEAMS = (16, 33, 64, 100, 128, 255, 256)


@pytest.mark.parametrize("P", LARGE_TEAMS)
def test_restatement_matches_reference_large_teams(rs, ref, P):
    """Every (algorithm, op) at P members, three type-table entries each
    (drawn per P), element counts on both sides of the Rabenseifner block
    boundaries (N < p2s, N not a multiple of p2s)."""
    rng = np.random.default_rng(1000 + P)
    for algo in oracle.ALGOS:
        for op in oracle.OPS:
            names = list(oracle.reduce_types(op))
            for tname in rng.choice(names, size=3, replace=False):
                dt = oracle.SHMEM_TYPES[tname]
                if algo == "binomial" and dt.startswith(("float", "complex")):
                    continue  # arrival-order dependent in the reference
                N = int(rng.choice([int(rng.integers(1, P)), int(rng.integers(P, 4 * P + 7))]))
                x = gen.random_values(oracle.NP[dt], P, N, int(rng.integers(1 << 30)))
                got = rs.reduce(algo, op, x)
                want, _ = ref.reduce(algo, op, x, tname=str(tname))
                assert value_bytes(got) == value_bytes(want), (algo, op, tname, P, N)


@pytest.mark.parametrize("P", (100, 128, 255, 256))
def test_restatement_matches_reference_special_minmax_large(rs, ref, P):
    """NaN and mixed-sign zeros at large P: rec_dbl leaves member-dependent
    bits, Rabenseifner block-dependent bits; both must match per member."""
    for dt, tname in ((np.float32, "float"), (np.float64, "double")):
        x = gen.special_minmax(dt, P, 3 * P + 5, P)
        for algo in ("rec_dbl", "rabenseifner", "rabenseifner2", "linear"):
            for op in ("min", "max"):
                want, _ = ref.reduce(algo, op, x, tname=tname)
                assert rs.reduce(algo, op, x).tobytes() == want.tobytes(), (algo, op, tname, P)


def test_restatement_matches_reference_config2_shape(rs, ref):
    """The headline shape itself: 64 members x 2^20 elements, f32 SUM
    N(0,1) in all three butterfly orders, f64 MAX U(+-1e6), i64 XOR."""
    P, N = 64, 1 << 20
    f32 = gen.normal(np.float32, P, N, 1)
    for algo in ("rec_dbl", "rabenseifner", "rabenseifner2"):
        want, _ = ref.reduce(algo, "sum", f32)
        assert rs.reduce(algo, "sum", f32).tobytes() == want.tobytes(), algo
    f64 = gen.uniform(np.float64, P, N, 2, -1e6, 1e6)
    want, _ = ref.reduce("rabenseifner", "max", f64)
    assert rs.reduce("rabenseifner", "max", f64).tobytes() == want.tobytes()
    i64 = gen.uniform_int(np.int64, P, N, 3)
    want, _ = ref.reduce("rec_dbl", "xor", i64)
    assert rs.reduce("rec_dbl", "xor", i64).tobytes() == want.tobytes()


def test_restatement_matches_reference_config3_shape(rs, ref):
    """The data-movement shapes at 128 members: fcollect64 of 4096 int64
    (the default bruck_inplace), alltoallmem of 64 KiB blocks and alltoalls64
    with dst 2, sst 3 over 4096 elements per pair (shift_exchange_barrier)."""
    P = 128
    x = gen.uniform_int(np.int64, P, 4096, 1)
    out = np.zeros((P, P * 4096), np.int64)
    ref.run(oracle.K_SIZED, "shcoll_fcollect64_bruck_inplace", x, out, nelems=4096)
    assert rs.fcollect(x).tobytes() == out.tobytes()
    x = gen.uniform_int(np.uint8, P, P * 65536, 2)
    out = np.zeros_like(x)
    ref.run(oracle.K_TEAM_COPY, "shcoll_alltoallmem_shift_exchange_barrier", x, out,
            nelems=65536)
    assert rs.alltoall(x).tobytes() == out.tobytes()
    del x, out
    n = 4096
    x = gen.uniform_int(np.int64, P, P * n * 3, 3)
    d0 = gen.uniform_int(np.int64, P, P * n * 2, 4)
    out = d0.copy()
    ref.run(oracle.K_ALLTOALLS_SIZED, "shcoll_alltoalls64_shift_exchange_barrier", x, out,
            nelems=n, a=2, b=3)
    assert rs.alltoalls(x, d0, 2, 3, n).tobytes() == out.tobytes()
