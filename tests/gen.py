"""Seeded synthetic inputs with the shapes and value distributions of the
benchmark configurations (there is no public dataset for this path)."""
import numpy as np

M64 = (1 << 64) - 1


def splitmix64(x):
    """Per-PE seed derivation: seed(pe) = splitmix64(master ^ pe)."""
    x = (x + 0x9E3779B97F4A7C15) & M64
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def pe_rng(master, pe):
    return np.random.default_rng(splitmix64(master ^ pe))


def uniform_int(dtype, npes, n, master, lo=None, hi=None):
    dt = np.dtype(dtype)
    info = np.iinfo(dt)
    lo = info.min if lo is None else lo
    hi = info.max if hi is None else hi
    return np.stack([pe_rng(master, p).integers(lo, hi, size=n, dtype=dt, endpoint=True)
                     for p in range(npes)]) if npes else np.zeros((0, n), dt)


def normal(dtype, npes, n, master):
    return np.stack([pe_rng(master, p).standard_normal(n).astype(dtype) for p in range(npes)])


def uniform(dtype, npes, n, master, lo, hi):
    return np.stack([pe_rng(master, p).uniform(lo, hi, n).astype(dtype) for p in range(npes)])


def random_values(dtype, npes, n, master):
    """Full-range values of any reduce dtype."""
    dt = np.dtype(dtype)
    if dt.kind in "iu":
        return uniform_int(dt, npes, n, master)
    if dt.kind == "c":
        re = normal(np.float64, npes, n, master)
        im = normal(np.float64, npes, n, master + 1)
        return (re + 1j * im).astype(dt)
    return normal(dt, npes, n, master)


def config1_inputs(npes=8, n_reduce=1024, n_fc=256, master=0xC0FFEE):
    """Config 1: int32 sum_reduce input uniform in [-1000, 1000] per PE seed;
    fcollect64 input value = pe * 2^32 + index."""
    x = uniform_int(np.int32, npes, n_reduce, master, -1000, 1000)
    fc = (np.arange(npes, dtype=np.int64)[:, None] << 32) | np.arange(n_fc, dtype=np.int64)[None, :]
    return x, fc


def special_minmax(dtype, npes, n, seed):
    """Floats where MIN/MAX depend on operand order: N(0,1) values with
    about 1/5 each +0 and -0, and 10 % NaNs with distinct payloads."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((npes, n)).astype(dtype)
    pick = rng.integers(0, 5, size=(npes, n))
    x[pick == 0] = 0.0
    x[pick == 1] = -0.0
    m = rng.random((npes, n)) < 0.1
    x[m] = np.nan
    bits = x.view(np.uint32 if np.dtype(dtype).itemsize == 4 else np.uint64)
    bits[m] |= rng.integers(1, 1 << 20, size=m.sum()).astype(bits.dtype)
    return x
