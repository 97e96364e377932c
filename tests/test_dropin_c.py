"""A C++ program written against include/talsh.h alone builds, links libtalsh.so
and runs the reference's test_talsh_c flow on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.gpu
def test_cxx_caller(built, tmp_path):
    exe = tmp_path / "test_talsh_c"
    lib_dir = os.path.join(ROOT, "tal_sh_b200")
    subprocess.run(["g++", "-O2", "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "c", "test_talsh_c.cpp"),
                    "-o", str(exe), "-L", lib_dir, "-ltalsh", "-Wl,-rpath," + lib_dir], check=True)
    p = subprocess.run([str(exe)], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=300)
    assert p.returncode == 0 and "PASS" in p.stdout, p.stdout
