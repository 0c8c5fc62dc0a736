"""Build the in-tree CUDA extension ``_tc_b200.so`` for sm_100a with nvcc.

The library is a plain C-ABI shared object (no torch types in its
signatures); ``torchannel_b200._lib`` loads it with ctypes.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "tc_capi.cu")
OUT = os.path.join(HERE, "_tc_b200.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr"]


def sources():
    d = os.path.join(HERE, "csrc")
    return [os.path.join(d, f) for f in sorted(os.listdir(d))] + [
        os.path.join(os.path.dirname(HERE), "include", "torchannel_b200.h")]


# The bounds-checked build: every checked global access of the step kernels
# compares its index with its buffer's extent and records a violation instead
# of making it (tc_bounds_error); slower, for tests.
CHECKED_OUT = os.path.join(HERE, "_tc_b200_check.so")


def needs_build(out=OUT):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in sources())


def build(force=False, verbose=False, extra=(), out=OUT):
    if not force and not needs_build(out):
        return out
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *NVCC_FLAGS, *extra, SRC, "-o", out + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(out + ".tmp", out)
    return out


def build_checked(force=False, verbose=False):
    return build(force=force, verbose=verbose, extra=["-DTC_BOUNDS_CHECK"], out=CHECKED_OUT)


if __name__ == "__main__":
    if "--checked" in sys.argv:
        print(build_checked(force="--force" in sys.argv, verbose=True))
    else:
        build(force="--force" in sys.argv, verbose=True,
              extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else [])
        print(OUT)
