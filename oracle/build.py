"""TEST INFRASTRUCTURE (oracle). Builds the CPU oracle and, where a reference
checkout exists, the compiled reference shaders.

  oracle/_build/liboracle.so     <- oracle.cpp + oracle_host.cpp (OpenMP)
  oracle/_ref/libretrocam_ref.so <- build_ref.py (reference shader source)

Both are checkers and the CPU baseline; the product never links them.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
BUILD_DIR = os.path.join(HERE, "_build")
ORACLE_LIB = os.path.join(BUILD_DIR, "liboracle.so")
SOURCES = ["oracle.cpp", "oracle_host.cpp"]
HEADERS = ["oracle_host.h", "half_soft.h", "glsl_compat.h"]


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build_oracle(force: bool = False) -> str:
    deps = [os.path.join(HERE, f) for f in SOURCES + HEADERS]
    deps += [os.path.join(REPO, "include", f) for f in ("retrocam.h", "rc_exact_math.h")]
    if not force and not _stale(ORACLE_LIB, deps):
        return ORACLE_LIB
    os.makedirs(BUILD_DIR, exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O3", "-march=x86-64-v2", "-fopenmp", "-fwrapv",
           "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-Wall",
           "-Wno-unused-function", "-I", HERE, "-I", os.path.join(REPO, "include")]
    cmd += [os.path.join(HERE, f) for f in SOURCES]
    cmd += ["-o", ORACLE_LIB + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(ORACLE_LIB + ".tmp", ORACLE_LIB)
    return ORACLE_LIB


def build_all(force: bool = False) -> dict:
    out = {"oracle": build_oracle(force)}
    sys.path.insert(0, HERE)
    try:
        import build_ref  # noqa: E402
        out["ref"] = build_ref.build(quiet=True)
    finally:
        sys.path.pop(0)
    return out


if __name__ == "__main__":
    print(build_all(force="--force" in sys.argv))
