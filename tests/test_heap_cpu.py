"""The symmetric-heap allocator's bookkeeping (osss-ucx_b200/csrc/
heap_core.cuh), built for the host from the same source the device runs,
against its invariants under seeded random allocation and free sequences
(tests/c/heap_model.cu): exact tiling, immediate merging, class lists and
bitmaps, no overlap, alignment, refusal only without room, exhaustion and
recovery.  Needs nvcc (no GPU)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


@pytest.fixture(scope="module")
def model(tmp_path_factory):
    if not (os.path.exists(NVCC) or shutil.which("nvcc")):
        pytest.skip("nvcc is not available")
    exe = str(tmp_path_factory.mktemp("heap") / "heap_model")
    subprocess.run([NVCC if os.path.exists(NVCC) else "nvcc", "-O2", "-std=c++17",
                    "-gencode", "arch=compute_100a,code=sm_100a", "-x", "cu",
                    "-I" + os.path.join(ROOT, "osss-ucx_b200", "csrc"),
                    os.path.join(ROOT, "tests", "c", "heap_model.cu"), "-o", exe],
                   check=True, capture_output=True)
    return exe


@pytest.mark.parametrize("seed", [1, 2, 3, 0xC0FFEE, 987654321])
def test_allocator_invariants(model, seed):
    r = subprocess.run([model, str(seed)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
