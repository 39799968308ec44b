"""In-tree build of the two native libraries.

* libbsgpu.so  -- the sm_100a engine (nvcc, -gencode arch=compute_100a,code=sm_100a)
* libbsghost.so -- the CPU table builder (g++)

Both land next to this file so they travel with the source tree.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _newer(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build_host(force=False, verbose=False):
    out = os.path.join(HERE, "libbsghost.so")
    srcs = [os.path.join(HERE, "host", "bsg_tables_build.cpp")]
    deps = srcs + glob.glob(os.path.join(ROOT, "include", "*.h"))
    if force or _newer(out, deps):
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I" + os.path.join(ROOT, "include")] + srcs + ["-o", out]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return out


def build_gpu(force=False, verbose=False, ptxas_verbose=False):
    out = os.path.join(HERE, "libbsgpu.so")
    srcs = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
    deps = srcs + glob.glob(os.path.join(HERE, "csrc", "*.h")) + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) \
        + glob.glob(os.path.join(ROOT, "include", "*.h"))
    if force or _newer(out, deps):
        cmd = [NVCC] + ARCH + ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-shared",
                               "-cudart", "static", "-I" + os.path.join(ROOT, "include")]
        if ptxas_verbose:
            cmd += ["-Xptxas", "-v"]
        cmd += srcs + ["-o", out]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return out


def build_all(force=False, verbose=False):
    return build_host(force, verbose), build_gpu(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose=True)
