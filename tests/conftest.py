import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "osss-ucx_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

# Heap used by the GPU tests: TEST_NPES PEs x TEST_HEAP bytes each.
TEST_NPES = 256
TEST_HEAP = 24 << 20


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def rs():
    import oracle
    return oracle.Restatement()


@pytest.fixture(scope="session")
def ref():
    import oracle
    if not oracle.Reference.available:
        pytest.skip("reference build oracle/_ref is absent (needs the reference tree)")
    return oracle.Reference()


@pytest.fixture(scope="session")
def B():
    """The engine, initialised once per test session on cuda:0."""
    sys.path.insert(0, ROOT)
    import __graft_entry__
    __graft_entry__.build_library()
    import b200shm
    if not b200shm.initialized():
        b200shm.init(TEST_NPES, TEST_HEAP)
    return b200shm


@pytest.fixture()
def heap(B):
    """Symmetric allocations that are freed after the test."""
    offs = []

    def alloc(nbytes):
        o = B.malloc(nbytes)
        offs.append(o)
        return o
    yield alloc
    for o in offs:
        B.free(o)
