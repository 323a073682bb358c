"""Builds retrocam_b200/_lib/libretrocam.so for sm_100a.

  kernels.cu, wavefront.cu  x2
                  -DRC_EXACT=1 -fmad=false  (bit-exact math, rc::exact)
                  -DRC_EXACT=0 -prec-div=false  (fast math, rc::fast: FMA
                  contraction, the approximate divide within 2 ulp)
  api.cu          C ABI, device half
  noalloc.cu      allocation-free à-trous entry point
  post_vhs.cu     the VHS chain (exact-math flags in both modes)
  kpcnn.cu        learned denoiser (tcgen05 BF16 convolutions)
  host_scene.cpp  C ABI, host half (-ffp-contract=off: Java float rules)

The CUDA runtime is linked statically so the library needs only the driver.
ptxas statistics (registers, spills, stack) go to _build/ptxas.log.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libretrocam.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "nvcc")


def _deps():
    out = []
    for d in (CSRC, os.path.join(REPO, "include")):
        for f in sorted(os.listdir(d)):
            if f.endswith((".cu", ".cuh", ".h", ".cpp", ".hpp")):
                out.append(os.path.join(d, f))
    return out + [os.path.abspath(__file__)]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, log=None):
    p = subprocess.run(cmd, capture_output=True, text=True)
    if log is not None:
        log.write(" ".join(cmd) + "\n" + p.stdout + p.stderr + "\n")
    if p.returncode != 0:
        sys.stderr.write(p.stdout + p.stderr)
        raise RuntimeError("command failed: " + " ".join(cmd[:6]) + " ...")
    return p


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale(LIB, _deps()):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    inc = ["-I", os.path.join(REPO, "include"), "-I", CSRC]
    common = [NVCC] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
                              "-Xptxas", "-v"] + inc
    objs = []
    with open(os.path.join(BUILD, "ptxas.log"), "w") as log:
        for name, flags in (("kernels_exact", ["-DRC_EXACT=1", "-fmad=false", "-prec-div=true",
                                               "-prec-sqrt=true", "-ftz=false"]),
                            ("kernels_fast", ["-DRC_EXACT=0", "-fmad=true", "-prec-div=false"])):
            for src in ("kernels", "wavefront"):
                o = os.path.join(BUILD, f"{src}_{name.split('_')[1]}.o")
                _run(common + flags + ["-c", os.path.join(CSRC, src + ".cu"), "-o", o], log)
                objs.append(o)
        for name in ("api", "noalloc", "kpcnn", "peak"):
            o = os.path.join(BUILD, name + ".o")
            _run(common + ["-c", os.path.join(CSRC, name + ".cu"), "-o", o], log)
            objs.append(o)
        # the VHS chain: exact arithmetic in every math mode
        o = os.path.join(BUILD, "post_vhs.o")
        _run(common + ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false", "-c",
                       os.path.join(CSRC, "post_vhs.cu"), "-o", o], log)
        objs.append(o)
        o = os.path.join(BUILD, "host_scene.o")
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall"] + inc +
             ["-c", os.path.join(CSRC, "host_scene.cpp"), "-o", o], log)
        objs.append(o)
        _run([NVCC] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs, log)
    os.replace(LIB + ".tmp", LIB)
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
