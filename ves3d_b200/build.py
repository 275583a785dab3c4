"""Build the ves3d_b200 CUDA library in-tree for sm_100a (nvcc, no JIT)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libves3d_b200.so")
# the benchmark's FMA-throughput probe, a separate library (not part of the product)
PEAK_LIB = os.path.join(HERE, "libves3d_peak.so")
PEAK_SOURCE = "peak_probe.cu"
SOURCES = ["sh_tables.cc", "sht_kernels.cu", "singular_kernels.cu", "direct_kernels.cu", "far_kernels.cu", "build_kernels.cu", "stokes_velocity.cu",
           "noalloc.cu", "geometry_kernels.cu", "bicgstab.cu", "mlp.cu", "device_prims.cu",
           "vtk_output.cu", "near_kernels.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared", "-Wno-deprecated-gpu-targets"]


# cuSOLVER: dense LU of the self-block preconditioner of the implicit solve
LIBS = ["-lcusolver", "-lcublas"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def sources():
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "ves3d_b200.h"))
    return srcs, deps


def _stale(out, deps):
    return not os.path.exists(out) or os.path.getmtime(out) < max(os.path.getmtime(d) for d in deps)


def build(force=False, verbose=False):
    srcs, deps = sources()
    peak_src = os.path.join(CSRC, PEAK_SOURCE)
    if force or _stale(PEAK_LIB, [peak_src]):
        cmd = [_nvcc()] + NVCC_FLAGS + ["-o", PEAK_LIB, peak_src]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd, cwd=CSRC)
    if not force and not _stale(LIB, deps):
        return LIB
    cmd = [_nvcc()] + NVCC_FLAGS + ["-o", LIB] + srcs + LIBS
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd, cwd=CSRC)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
