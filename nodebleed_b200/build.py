"""Build the native libraries of nodebleed_b200 in-tree.

    libnbhost.so  host C: render-data bridge, BVH8 build, synthetic scenes
    libnbgpu.so   CUDA sm_100a kernels + the rendgpu C ABI

`python -m nodebleed_b200.build` builds both; nvcc cross-compiles without a
GPU.  The BVH8 build file is compiled with the reference renderer's own float
flags (-O3 -mavx2 -mfma -ffast-math, Makefile:5-10 of nodebleed) because its
split decisions, and so the node bytes, depend on how the area sums are
contracted.  The CUDA file is compiled with -fmad=false: every fused
multiply-add in it is written out, so the shading arithmetic matches the CPU
oracle bit for bit.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _newer(out, srcs):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(s) <= t for s in srcs)


def build_host(force=False):
    out = os.path.join(HERE, "libnbhost.so")
    scene = os.path.join(CSRC, "host", "scene.c")
    bvh = os.path.join(CSRC, "host", "bvh8.c")
    gltf = os.path.join(CSRC, "host", "nb_gltf.c")
    hdrs = [os.path.join(CSRC, "host", h) for h in ("nb_host.h", "nb_rdata.h")]
    if not force and _newer(out, [scene, bvh, gltf] + hdrs):
        return out
    tmp = os.path.join(HERE, "_build")
    os.makedirs(tmp, exist_ok=True)
    o1 = os.path.join(tmp, "scene.o")
    o2 = os.path.join(tmp, "bvh8.o")
    _run(["gcc", "-std=gnu11", "-O2", "-fPIC", "-Wall", "-Wextra",
          "-c", scene, "-o", o1])
    _run(["gcc", "-std=gnu11", "-O3", "-mavx2", "-mfma", "-ffast-math",
          "-fPIC", "-Wall", "-Wextra", "-c", bvh, "-o", o2])
    o3 = os.path.join(tmp, "nb_gltf.o")
    _run(["gcc", "-std=gnu11", "-O2", "-fPIC", "-Wall", "-Wextra",
          "-c", gltf, "-o", o3])
    _run(["gcc", "-shared", "-o", out, o1, o2, o3, "-lm"])
    return out


def build_gpu(force=False):
    out = os.path.join(HERE, "libnbgpu.so")
    cu = os.path.join(CSRC, "rendgpu.cu")
    cpp = os.path.join(CSRC, "layout.cpp")
    cpp2 = os.path.join(CSRC, "blas_build.cpp")
    deps = [cu, cpp, cpp2] + [os.path.join(CSRC, f) for f in
                        ("trace.cuh", "kernels.cuh", "nrc.cuh", "gpulayout.h",
                         "layout.hpp", "qnode.h", "tlas_build.cuh", "tlas_cta.cuh",
                         os.path.join("host", "nb_rdata.h"))]
    deps.append(os.path.join(ROOT, "include", "rendgpu.h"))
    if not force and _newer(out, deps):
        return out
    tmp = os.path.join(HERE, "_build")
    os.makedirs(tmp, exist_ok=True)
    o1 = os.path.join(tmp, "layout.o")
    o2 = os.path.join(tmp, "rendgpu.o")
    o3 = os.path.join(tmp, "blas_build.o")
    _run(["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", "-I", CSRC,
          "-c", cpp, "-o", o1])
    _run(["g++", "-std=c++17", "-O2", "-fPIC", "-Wall", "-I", CSRC,
          "-c", cpp2, "-o", o3])
    _run([NVCC, "-std=c++17", "-O3", "-lineinfo", "-fmad=false",
          "-Xptxas", "-v", "-Xcompiler", "-fPIC", "-I", CSRC] + ARCH +
         ["-c", cu, "-o", o2])
    _run([NVCC, "-shared", "-o", out, o1, o3, o2] + ARCH)
    return out


def build(force=False):
    return build_host(force), build_gpu(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
