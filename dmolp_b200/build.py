"""In-tree build of the native libraries (no JIT cache: the built .so files sit next to the sources).

    python -m dmolp_b200.build            # everything that is out of date

Products:
  dmolp_b200/lib/libdmolp_b200.so   CUDA kernels (sm_100a) + the C-ABI in include/dmolp_b200.h
  dmolp_b200/lib/libdmolp_dropin.so the reference's C++ entry points (run_phase1, run_phase2, ...) over the C-ABI
  dmolp_b200/lib/libdmolp_gen.so    seeded graph generators (host C++/OpenMP)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "lib")
INCLUDE = os.path.join(ROOT, "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
CXX = os.environ.get("DMOLP_CXX", "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++")

# Strict IEEE double on the host (no -ffast-math, no FMA contraction): the penalty arithmetic must follow
# the source's evaluation order; -march is fixed so the prebuilt library runs on any AVX2 host.
HOST_FLAGS = ["-std=c++17", "-O3", "-march=x86-64-v3", "-fno-fast-math", "-ffp-contract=off", "-fPIC", "-Wall",
              "-Wno-unused-function"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", *GENCODE, "-Xcompiler", "-fPIC,-fno-fast-math,-ffp-contract=off",
              "--expt-relaxed-constexpr", "-Xptxas", "-v"]

CUDA_SOURCES = ["dmolp_cabi.cu", "lp_kernels.cu", "seed_kernels.cu", "select_kernels.cu", "adjtext.cpp",
                "noalloc.cu", "ingest.cu", "hubsort.cpp", "batch_kernels.cu", "batch_cabi.cu", "batch_p1.cu", "mpnn_kernels.cu", "mpnn_cabi.cu"]
CUDA_HEADERS = ["common.cuh", "device_state.cuh", "kernels.cuh", "lp_device.cuh", "batch.cuh", "mpnn.cuh", "umma.cuh", "ingest.cuh"]
DROPIN_SOURCES = ["dropin.cpp"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def _run(cmd: list[str], log: list[str] | None = None) -> None:
    p = subprocess.run(cmd, capture_output=True, text=True)
    if log is not None:
        log.append(p.stdout + p.stderr)
    if p.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + p.stdout + p.stderr)
        raise RuntimeError(f"build step failed: {cmd[0]} (exit {p.returncode})")


def build_gen(force: bool = False) -> str:
    out = os.path.join(LIB, "libdmolp_gen.so")
    deps = [os.path.join(CSRC, "graphgen.cpp"), os.path.join(CSRC, "graphgen.h")]
    if force or _newer(out, deps):
        os.makedirs(LIB, exist_ok=True)
        _run([CXX, *HOST_FLAGS, "-fopenmp", "-shared", "-o", out, deps[0]])
    return out


def build_cuda(force: bool = False, ptxas_log: list[str] | None = None) -> str:
    out = os.path.join(LIB, "libdmolp_b200.so")
    srcs = [os.path.join(CSRC, s) for s in CUDA_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    deps = srcs + [os.path.join(CSRC, h) for h in CUDA_HEADERS] + [os.path.join(INCLUDE, "dmolp_b200.h")]
    if force or _newer(out, deps):
        os.makedirs(LIB, exist_ok=True)
        objdir = os.path.join(LIB, "obj")
        os.makedirs(objdir, exist_ok=True)
        objs = []
        for s in srcs:
            o = os.path.join(objdir, os.path.basename(s) + ".o")
            if s.endswith(".cpp"):
                _run([CXX, *HOST_FLAGS, "-fopenmp", "-I", INCLUDE, "-I", CSRC, "-c", s, "-o", o])
            else:
                _run([NVCC, *NVCC_FLAGS, "-Xcompiler", "-fopenmp", "-I", INCLUDE, "-I", CSRC, "-c", s, "-o", o],
                     ptxas_log)
            objs.append(o)
        _run([NVCC, "-shared", *GENCODE, "-o", out, *objs, "-lcudart_static", "-lrt", "-lpthread", "-ldl",
              "-Xcompiler", "-fopenmp", "-Xlinker", "--exclude-libs,ALL"])
    return out


def build_dropin(force: bool = False) -> str:
    out = os.path.join(LIB, "libdmolp_dropin.so")
    srcs = [os.path.join(CSRC, s) for s in DROPIN_SOURCES]
    deps = srcs + [os.path.join(CSRC, "dropin_types.hpp"),
                   os.path.join(INCLUDE, "dmolp_b200.h"), os.path.join(LIB, "libdmolp_b200.so")]
    if force or _newer(out, deps):
        cuda_lib = os.path.join(CUDA_HOME, "lib64")
        _run([CXX, *HOST_FLAGS, "-fopenmp", "-shared", "-I", INCLUDE, "-I", CSRC, "-I", os.path.join(CUDA_HOME, "include"),
              "-o", out, *srcs, "-L", LIB, "-ldmolp_b200", "-L", cuda_lib, "-lcudart", "-Wl,-rpath,$ORIGIN",
              "-Wl,-rpath," + cuda_lib])
    return out


def build_oracle() -> None:
    """The checker (oracle/): the CPU restatement always; the reference harness when the reference tree exists."""
    make = shutil.which("make")
    if make is None:
        raise RuntimeError("make not found")
    _run([make, "-s", "-C", os.path.join(ROOT, "oracle"), "-j8"])


def build_all(force: bool = False) -> None:
    build_gen(force)
    build_cuda(force)
    build_dropin(force)
    build_oracle()


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built:", ", ".join(sorted(f for f in os.listdir(LIB) if f.endswith(".so"))))
