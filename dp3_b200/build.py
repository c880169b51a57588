"""Builds the in-tree native libraries of dp3_b200.

  libddsolve_b200.so   CUDA solver (sm_100a) + C ABI (include/ddsolve_b200.h)
  libddwarm_b200.so    learned warm start on the tensor cores (sm_100a) + C ABI
                       (include/ddwarm_b200.h)
  libdp3b200_synth.so  seeded synthetic-observation generator (host C++)

Both are built with explicit nvcc / g++ command lines (no JIT cache), so the
shared objects live next to the sources and travel with the repository tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")

SOLVER_SO = os.path.join(HERE, "libddsolve_b200.so")
SYNTH_SO = os.path.join(HERE, "libdp3b200_synth.so")
WARM_SO = os.path.join(HERE, "libddwarm_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def build_solver(force=False, verbose_ptxas=False):
    srcs = [os.path.join(CSRC, "ddsolve.cu"),
            os.path.join(INCLUDE, "ddsolve_b200.h")]
    if not force and not _stale(SOLVER_SO, srcs):
        return SOLVER_SO
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
           "-I", INCLUDE, "-o", SOLVER_SO, srcs[0], "-lcudart"]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    _run(cmd)
    return SOLVER_SO


def build_warm(force=False, verbose_ptxas=False):
    srcs = [os.path.join(CSRC, "warmstart.cu"),
            os.path.join(INCLUDE, "ddwarm_b200.h")]
    if not force and not _stale(WARM_SO, srcs):
        return WARM_SO
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
           "-I", INCLUDE, "-o", WARM_SO, srcs[0], "-lcudart"]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    _run(cmd)
    return WARM_SO


def build_synth(force=False):
    srcs = [os.path.join(CSRC, "synth.cc"), os.path.join(CSRC, "synth.h")]
    if not force and not _stale(SYNTH_SO, srcs):
        return SYNTH_SO
    _run(["g++", "-std=c++17", "-O3", "-march=x86-64-v3", "-fPIC", "-shared",
          "-fopenmp", "-Wall", "-o", SYNTH_SO, srcs[0]])
    return SYNTH_SO


def build_all(force=False):
    build_solver(force)
    build_warm(force)
    build_synth(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
