"""Every function the reference's public headers declare (include/shmem.h
and include/shmem/*.h, after the preprocessor expands their type tables)
is exported by libshmem_b200.so under the same name, so a program built
against the reference's headers links against this library.  Runs where
the reference tree is present (found as the oracle finds it), on the CPU;
skipped elsewhere."""
import os
import re
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

# a static inline helper of the reference's generics header, not a library symbol
NOT_LIBRARY = {"shmem_generics_nomatch"}


def reference_api_names(tree, tmp):
    inc = os.path.join(tmp, "inc")
    shutil.copytree(os.path.join(tree, "include"), inc)
    # configure fills defs_subst.h from its template; any values do here
    with open(os.path.join(inc, "shmem", "defs_subst.h.in")) as f:
        text = re.sub(r'"?@[A-Z_]+@"?', "1", f.read())
    with open(os.path.join(inc, "shmem", "defs_subst.h"), "w") as f:
        f.write(text)
    pp = subprocess.run(["gcc", "-E", "-P", "-x", "c", "-std=gnu11", "-I", inc,
                         os.path.join(inc, "shmem.h")], capture_output=True, text=True, check=True)
    return set(re.findall(
        r"\b((?:shmem|shmemx|pshmem|shmalloc|shfree|shrealloc|shmemalign|start_pes|_my_pe|"
        r"_num_pes)[A-Za-z0-9_]*)\s*\(", pp.stdout))


def test_every_reference_api_function_is_exported(tmp_path):
    import ctypes
    import oracle
    tree = oracle.reference_tree()
    if tree is None:
        pytest.skip("the reference tree is absent")
    import __graft_entry__
    __graft_entry__.build_library()
    names = reference_api_names(tree, str(tmp_path))
    assert len(names) > 1500
    lib = ctypes.CDLL(os.path.join(ROOT, "osss-ucx_b200", "lib", "libshmem_b200.so"))
    missing = sorted(n for n in names - NOT_LIBRARY if not hasattr(lib, n))
    assert not missing, (len(missing), missing[:30])
