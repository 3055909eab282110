"""Build the CUDA library of the pbpic B200 step in-tree.

`python -m pbpic_b200.build` compiles pbpic_b200/csrc/pbpic_api.cu and
pbpic_diff.cu (which include the kernels) for sm_100a into
pbpic_b200/libpbpic.so, and the C++
host driver (the reference time loop on the C ABI) into
pbpic_b200/pic2d_driver. Nothing is compiled at import time.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libpbpic.so")
DRIVER = os.path.join(HERE, "pic2d_driver")

NVCC_FLAGS = [
    "-O3", "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler", "-fPIC,-ffp-contract=off",
    "-Xptxas", "-warn-spills",
]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd))
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def sources():
    out = [os.path.join(ROOT, "include", "pbpic.h")]
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cuh", ".h", ".cpp")):
            out.append(os.path.join(CSRC, f))
    return out


def build(force=False, verbose=False, ptxas_verbose=False):
    src = sources()
    if force or _stale(LIB, src):
        flags = list(NVCC_FLAGS)
        if ptxas_verbose:
            flags += ["-Xptxas", "-v"]
        cus = [os.path.join(CSRC, f) for f in ("pbpic_api.cu", "pbpic_diff.cu")]
        _run([nvcc(), *flags, "-shared", "-o", LIB, *cus], verbose)
    drv_src = os.path.join(CSRC, "pic2d_driver.cpp")
    if os.path.exists(drv_src) and (force or _stale(DRIVER, src + [LIB])):
        _run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-o", DRIVER, drv_src,
              "-L", HERE, "-lpbpic", "-Wl,-rpath,$ORIGIN"], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_verbose="-v" in sys.argv)
