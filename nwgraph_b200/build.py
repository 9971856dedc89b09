"""In-tree build of the native libraries (sm_100a only).

    python -m nwgraph_b200.build

* ``libnwgpu.so``  -- CUDA kernels + the C ABI of include/nwgpu.h (nvcc, sm_100a)
* ``libnwgen.so``  -- seeded synthetic graph builder, include/nwgraph_gen.h (g++)
* ``tests/cpp/dropin_test`` -- C++20 drop-in test program for the header layer
  include/nwgraph_gpu/page_rank.hpp (links libnwgpu.so)

The libraries are written next to this file so they travel with the source
tree; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SOURCES = ["api.cu", "api_ppr.cu", "pr_plain.cu", "pr_binned.cu", "graph_build.cu", "ppr_batched.cu", "pr_noalloc.cu", "devmem.cu", "pr_weighted.cu", "api_wpr.cu", "api_ragged.cu", "csr_build.cu", "api_tune.cu", "api_shard.cu", "pr_blocked.cu", "ragged_union.cu", "loaders.cpp"]


def _run(cmd, cwd=None):
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=cwd)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _deps(names):
    files = [os.path.join(CSRC, s) for s in names]
    files += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    files += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return files


def build_cuda(force=False, verbose_ptxas=False):
    target = os.path.join(HERE, "libnwgpu.so")
    if not force and not _stale(target, _deps(CUDA_SOURCES)):
        return target
    cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-Xlinker", "--exclude-libs,ALL", f"-I{INCLUDE}", "-o", target, *CUDA_SOURCES]
    if verbose_ptxas:
        cmd.insert(-len(CUDA_SOURCES) - 2, "-Xptxas=-v")
    _run(cmd, cwd=CSRC)
    return target


def build_gen(force=False):
    target = os.path.join(HERE, "libnwgen.so")
    src = [os.path.join(CSRC, "graphgen.cpp"), os.path.join(INCLUDE, "nwgraph_gen.h")]
    if not force and not _stale(target, src):
        return target
    _run([CXX, "-std=c++20", "-O3", "-march=x86-64-v3", "-fPIC", "-shared", "-pthread",
          "-Wl,--exclude-libs,ALL", "-o", target, src[0]])
    return target


def build_probe(force=False):
    """libnwprobe.so: the random-gather ceiling probe the benchmark reports beside the HBM roofline."""
    target = os.path.join(HERE, "libnwprobe.so")
    deps = _deps(["probe_gather.cu"])
    if not force and not _stale(target, deps):
        return target
    _run([NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-Xlinker",
          "--exclude-libs,ALL", "-o", target, "probe_gather.cu"], cwd=CSRC)
    return target


def build_dropin_test(force=False):
    """tests/cpp/dropin_test: the C++20 header layer over libnwgpu.so."""
    src = os.path.join(ROOT, "tests", "cpp", "dropin_test.cpp")
    target = os.path.join(ROOT, "tests", "cpp", "dropin_test")
    lib = os.path.join(HERE, "libnwgpu.so")
    deps = [src, lib, os.path.join(INCLUDE, "nwgraph_gpu", "page_rank.hpp"), os.path.join(INCLUDE, "nwgpu.h")]
    if not os.path.exists(src) or (not force and not _stale(target, deps)):
        return target
    _run([CXX, "-std=c++20", "-O2", "-pthread", f"-I{INCLUDE}", "-o", target, src, f"-L{HERE}", "-l:libnwgpu.so",
          "-Wl,-rpath,$ORIGIN/../../nwgraph_b200"])
    return target


def build_all(force=False):
    build_gen(force)
    build_cuda(force)
    build_probe(force)
    build_dropin_test(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
