"""Build libefs.so (the CUDA engine behind include/efs.h) in-tree for sm_100a.

The library is plain CUDA C++ with a C ABI: it links only cudart, so a
ctypes / N-API / cffi host can load it without PyTorch.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libefs.so")
SOURCES = ["efs_engine.cu"]
HEADERS = ["efs_kernels.cuh", "efs_fused.cuh", "efs_tma.cuh", "efs_batch.cuh", "efs_host.h", os.path.join("..", "..", "include", "efs.h")]

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-shared",
    "-Xptxas", "-v",
    "--expt-relaxed-constexpr",
]


def nvcc_path():
    cand = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = os.path.join(cand, "bin", "nvcc")
    return p if os.path.exists(p) else (shutil.which("nvcc") or "nvcc")


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [__file__]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    """Compile libefs.so if it is missing or older than its sources."""
    if not force and not _stale():
        return LIB
    cmd = [nvcc_path()] + NVCC_FLAGS + ["-I", os.path.join(ROOT, "include"), "-o", LIB + ".tmp"]
    cmd += [os.path.join(CSRC, s) for s in SOURCES]
    res = subprocess.run(cmd, capture_output=True, text=True)
    log = os.path.join(HERE, "build.log")
    with open(log, "w") as f:
        f.write(" ".join(cmd) + "\n" + res.stdout + res.stderr)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libefs.so (see %s)" % log)
    os.replace(LIB + ".tmp", LIB)
    if verbose:
        sys.stdout.write(res.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
