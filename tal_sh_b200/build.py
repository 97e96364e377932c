"""Builds the talsh-b200 shared library (libtalsh.so) in-tree for sm_100a.

Usage: python -m tal_sh_b200.build  (or tal_sh_b200.build.build_library()).
The library exports the TAL-SH C API (include/talsh.h) and the device-level
C ABI (include/talsh_b200.h).  CUDA runtime is linked statically, so the .so
has no dependency on a particular libcudart on the target machine.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libtalsh.so")
BUILD_DIR = os.path.join(ROOT, "_build", "talsh")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SOURCES = ["permute.cu", "elementwise.cu", "contract.cu", "diag.cu", "noalloc.cu", "ozaki.cu", "slice.cu"]
CXX_SOURCES = ["pattern.cpp", "runtime.cpp", "serve.cpp"]
COMMON = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC]


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _run(cmd):
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return proc.stdout


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force=False, verbose=False):
    """Compiles every source for sm_100a and links libtalsh.so; returns its path."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(INCLUDE, h) for h in os.listdir(INCLUDE)] + [
        os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith(".h")]
    objs = []
    for src in CUDA_SOURCES + CXX_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD_DIR, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path] + headers):
            cmd = [nvcc] + ARCH + COMMON + ["-lineinfo", "-diag-suppress", "177"]
            if src.endswith(".cpp"):
                cmd += ["-x", "c++"]
            cmd += ["-c", path, "-o", obj]
            out = _run(cmd)
            if verbose and out:
                print(out)
    if force or _stale(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread", "-ldl", "-lrt"])
    return LIB


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose=True))
