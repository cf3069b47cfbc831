"""Build ``libluna_b200.so`` in-tree for sm_100a with nvcc."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "luna_b200.cu")
OUT = os.path.join(HERE, "libluna_b200.so")
DEPS = [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))
        if f not in ("peaks.cu", "surrogate.cu")]
DEPS.append(os.path.join(HERE, "..", "include", "luna_b200.h"))

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in DEPS)


# FMA-throughput microbenchmark (the compute ceilings of the benchmark's roofline)
PEAKS_SRC = os.path.join(HERE, "csrc", "peaks.cu")
PEAKS_OUT = os.path.join(HERE, "libluna_peaks.so")
# the learned surrogate's training and inference kernels (include/luna_surrogate.h)
SG_SRC = os.path.join(HERE, "csrc", "surrogate.cu")
SG_DEPS = [SG_SRC, os.path.join(HERE, "csrc", "tc_gemm.cuh"), os.path.join(HERE, "csrc", "common.cuh"),
           os.path.join(HERE, "..", "include", "luna_surrogate.h")]
SG_OUT = os.path.join(HERE, "libluna_surrogate.so")


def _stale(out, deps):
    return not os.path.exists(out) or any(os.path.getmtime(d) > os.path.getmtime(out) for d in deps)


def build(force=False, verbose=False):
    nvcc = os.environ.get("NVCC", "nvcc")
    if force or _stale(PEAKS_OUT, [PEAKS_SRC]):
        subprocess.run([nvcc] + NVCC_FLAGS + ["-o", PEAKS_OUT, PEAKS_SRC], check=True)
    if force or _stale(SG_OUT, SG_DEPS):
        subprocess.run([nvcc] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", SG_OUT, SG_SRC],
                       check=True)
    if not force and up_to_date():
        return OUT
    cmd = [nvcc] + NVCC_FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-o", OUT, SRC]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
