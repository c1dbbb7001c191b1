"""Build the B200 library ``vlfeat_b200/lib/libvl.so`` with nvcc (sm_100a).

The library is a drop-in for VLFeat's ``libvl.so`` on the GMM / Fisher path:
it exports the reference's C API (``include/vl/*.h``) plus the extensions of
``include/vlb200.h``.  nvcc cross-compiles without a GPU.

    python -m vlfeat_b200.build          # incremental
    python -m vlfeat_b200.build --force  # rebuild everything
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT_DIR = os.path.join(PKG, "lib")
OBJ_DIR = os.path.join(ROOT, "_build", "obj")
LIB = os.path.join(OUT_DIR, "libvl.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
          "-I", os.path.join(ROOT, "include"), "-I", CSRC]
SOURCES = ["runtime.cpp", "gmm_api.cpp", "fisher_api.cpp", "fisher_plan.cpp", "k_exact.cu", "k_tc.cu", "k_noalloc.cu",
           "k_router.cu", "k_mlp.cu", "k_vlad.cu", "k_pca.cu", "k_kmeans.cu"]
HEADERS = ["common.h", "engine.h", "tc_common.cuh", "exact_math.cuh"]


def _newer(src: str, dst: str, deps) -> bool:
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.exists(p) and os.path.getmtime(p) > t for p in [src, *deps])


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    deps = [os.path.join(CSRC, h) for h in HEADERS]
    deps += [os.path.join(ROOT, "include", p) for p in ("vlb200.h", "vl/gmm.h", "vl/fisher.h", "vl/random.h", "vl/vlad.h", "vl/kmeans.h",
                                                          "vl/generic.h", "vl/host.h")]
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ_DIR, src + ".o")
        objs.append(o)
        if force or _newer(s, o, deps):
            cmd = [NVCC, *ARCH, *COMMON, "-c", s, "-o", o]
            if src.endswith(".cu"):
                cmd += ["-Xptxas", "-v"] if verbose else []
            else:
                cmd += ["-x", "cu"] if False else []
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
    if force or any(_newer(o, LIB, []) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static" if False else "-lcudart",
               "-Xlinker", "-soname,libvl.so", "-Xlinker", "-Bsymbolic"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    sys.exit(main())
