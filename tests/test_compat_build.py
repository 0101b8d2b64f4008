"""The reference's C++ call surface over the C ABI (include/bem/*.h,
libbem_compat.so): a consumer making the dense branch's calls in the
reference's call forms (tests/compat/dense_branch.cpp) compiles against these
headers alone and links against the two libraries.  CPU only: running it
needs a GPU."""
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(REPO, "bem-cpp_b200", "lib")


def test_dense_branch_consumer_builds_against_the_compat_surface(tmp_path):
    if not os.path.exists(os.path.join(LIB, "libbem_compat.so")):
        pytest.skip("libbem_compat.so not built")
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    exe = tmp_path / "dense_branch"
    cmd = [cxx, "-O1", "-std=c++17", "-Wall", "-Werror",
           "-I" + os.path.join(REPO, "include", "bem"), "-I" + os.path.join(REPO, "include"),
           "-o", str(exe), os.path.join(REPO, "tests", "compat", "dense_branch.cpp"),
           "-L" + LIB, "-Wl,-rpath," + LIB, "-lbem_compat", "-lbemdense"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert exe.exists()
