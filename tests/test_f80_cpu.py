"""The software x87 arithmetic behind the long double reductions
(osss-ucx_b200/csrc/f80.cuh), built for the host from the same source the
device runs, against this machine's own x87 long double: add, multiply and
the comparisons on every encoding class (normals, denormals,
pseudo-denormals, zeros, infinities, quiet and signalling NaNs, unnormals),
bit for bit (tests/c/f80_model.cpp).  Needs g++ on x86-64 (no GPU)."""
import os
import platform
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def model(tmp_path_factory):
    if platform.machine() not in ("x86_64", "AMD64") or not shutil.which("g++"):
        pytest.skip("needs g++ and an x87 long double")
    exe = str(tmp_path_factory.mktemp("f80") / "f80_model")
    subprocess.run(["g++", "-O2", "-std=c++17",
                    "-I" + os.path.join(ROOT, "osss-ucx_b200", "csrc"),
                    os.path.join(ROOT, "tests", "c", "f80_model.cpp"), "-o", exe],
                   check=True, capture_output=True)
    return exe


@pytest.mark.parametrize("seed", ["1", "0xC0FFEE", "987654321"])
def test_f80_matches_x87(model, seed):
    r = subprocess.run([model, "200000", seed], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("0 mismatches"), r.stdout + r.stderr
