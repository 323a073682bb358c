"""TEST INFRASTRUCTURE (oracle). Builds oracle/_ref/libretrocam_ref.so: the
reference's own hot-path shaders, compiled on the host.

The GLSL sources are read where they lie under the reference checkout
(pathtrace.comp, photon_trace.comp, photon_gather.comp,
post/atrous_denoise.frag, post/p00_normalize.frag, display.frag and the
fourteen VHS passes post/p01..p16), rewritten in memory by the
mechanical transforms below, wrapped in C++ namespaces on top of
oracle/glsl_compat.h, followed by oracle/ref_dispatch.inc (the dispatch loops
that stand in for glDispatchCompute / glDrawArrays), and piped to g++ on
stdin.  No transformed or original shader text is written to disk; only the
shared library lands in oracle/_ref/ (git-ignored; it travels with the
working tree to machines that have no reference checkout).

Transforms (each keeps the meaning of the GLSL statement):
  * drop `#version` and `layout(local_size...) in;`
  * `layout(std430, binding=N) [q] buffer B { T name[]; };` -> `T* name = nullptr;`
  * drop `layout(...)`, `readonly`, `writeonly`, `coherent`, leading `uniform`
  * top-level `in T v;` / `out T v;` -> `thread_local T v;`
  * parameters `inout T x` / `out T x` -> `T& x`
  * `T[N](a, b, ...)` array constructors -> `{a, b, ...}`
  * vector constructors with two or more `rand(` calls -> brace init, so the
    calls run left to right as GLSL 4.30 section 6.1.1 requires
  * swizzles `.rgb/.xyz` -> `.xyz()`, `.xy` -> `.xy()`, `.yz` -> `.yz()` (and
    `v.yz = e;` -> `v.set_yz(e);`), `.r/.g/.b` -> `.x/.y/.z`
  * floating literals get an `f` suffix (GLSL literals are single precision)
"""
from __future__ import annotations

import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def default_ref_root() -> str:
    """Where the reference checkout is looked for: $RETROCAM_REFERENCE, else a
    directory named `reference` beside this repository's root."""
    env = os.environ.get("RETROCAM_REFERENCE")
    if env:
        return env
    return os.path.join(os.path.dirname(REPO), "reference")

SHADER_DIR = os.path.join("src", "main", "resources", "shaders")
SHADERS = [
    ("pt", "pathtrace.comp"),
    ("phtrace", "photon_trace.comp"),
    ("phgather", "photon_gather.comp"),
    ("atrous", os.path.join("post", "atrous_denoise.frag")),
    ("p00", os.path.join("post", "p00_normalize.frag")),
    ("display", "display.frag"),
] + [(name.split("_")[0], os.path.join("post", name + ".frag")) for name in (
    "p01_downsample", "p02_chroma_res", "p03_color_matrix", "p04_dynamic_range", "p07_ccd_noise",
    "p08_ccd_smear", "p09_chroma_bleed", "p10_timebase", "p11_dot_crawl", "p12_dropout", "p13_headswitch",
    "p14_tracking", "p15_edge_enhance", "p16_interlace")]
OUT_DIR = os.path.join(HERE, "_ref")
OUT_LIB = os.path.join(OUT_DIR, "libretrocam_ref.so")
# timing variant: sin/cos/exp/log/pow from the host C library (not for parity)
OUT_LIB_LIBM = os.path.join(OUT_DIR, "libretrocam_ref_libm.so")


def _match_paren(s: str, open_idx: int) -> int:
    depth = 0
    for i in range(open_idx, len(s)):
        if s[i] == "(":
            depth += 1
        elif s[i] == ")":
            depth -= 1
            if depth == 0:
                return i
    raise ValueError("unbalanced parentheses")


def _replace_ctor_parens(src: str, pattern: str, want) -> str:
    out, pos = [], 0
    for m in re.finditer(pattern, src):
        if m.start() < pos:
            continue
        open_idx = m.end() - 1
        close_idx = _match_paren(src, open_idx)
        inner = src[open_idx + 1:close_idx]
        if want(m, inner):
            head = src[m.start():open_idx] if m.group(0).startswith(("vec", "ivec")) else ""
            out.append(src[pos:m.start()])
            out.append(head + "{" + inner + "}")
            pos = close_idx + 1
    out.append(src[pos:])
    return "".join(out)


def transform(src: str) -> str:
    s = re.sub(r"^\s*#version[^\n]*\n", "", src, flags=re.M)
    s = re.sub(r"layout\s*\(\s*local_size[^)]*\)\s*in\s*;", "", s)
    s = re.sub(
        r"layout\s*\(\s*std430[^)]*\)\s*(?:readonly|writeonly|coherent)?\s*buffer\s+\w+\s*"
        r"\{\s*(\w+)\s+(\w+)\s*\[\s*\]\s*;\s*\}\s*;",
        r"\1* \2 = nullptr;", s)
    s = re.sub(r"layout\s*\([^)]*\)\s*", "", s)
    s = re.sub(r"\b(?:readonly|writeonly|coherent)\s+", "", s)
    s = re.sub(r"^(\s*)uniform\s+", r"\1", s, flags=re.M)
    s = re.sub(r"^(in|out)\s+(\w+)\s+(\w+)\s*;", r"thread_local \2 \3;", s, flags=re.M)
    s = re.sub(r"\b(?:inout|out)\s+(\w+)\s+(\w+)", r"\1& \2", s)
    # float[5](...) -> {...}
    s = _replace_ctor_parens(s, r"\b(?:float|int)\s*\[\s*\d+\s*\]\s*\(",
                             lambda m, inner: True)
    # vecN(rand(..), rand(..)) -> vecN{...}
    s = _replace_ctor_parens(s, r"\b(?:vec[234])\s*\(",
                             lambda m, inner: inner.count("rand(") >= 2)
    s = re.sub(r"(\w+)\.yz\s*=\s*([^;]+);", r"\1.set_yz(\2);", s)   # swizzle write
    s = re.sub(r"\.yz\b(?!\()", ".yz()", s)
    s = re.sub(r"\.(?:rgb|xyz)\b", ".xyz()", s)
    s = re.sub(r"\.xy\b", ".xy()", s)
    s = re.sub(r"\.r\b", ".x", s)
    s = re.sub(r"\.g\b", ".y", s)
    s = re.sub(r"\.b\b", ".z", s)
    s = re.sub(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])",
               r"\1f", s)
    return s


def translation_unit(ref_root: str) -> str:
    parts = ['#include "glsl_compat.h"', '#include "retrocam.h"']
    for ns, rel in SHADERS:
        path = os.path.join(ref_root, SHADER_DIR, rel)
        with open(path, "r", encoding="utf-8") as f:
            body = transform(f.read())
        prologue = ("thread_local uvec3 gl_GlobalInvocationID;\n" if rel.endswith(".comp")
                    else "thread_local vec4 gl_FragCoord;\n")
        parts.append(f"namespace glsl {{ namespace {ns} {{\n{prologue}#line 1 \"{rel}\"\n{body}\n}} }}")
    with open(os.path.join(HERE, "ref_dispatch.inc"), "r", encoding="utf-8") as f:
        parts.append('#line 1 "ref_dispatch.inc"\n' + f.read())
    return "\n".join(parts)


def build(ref_root: str | None = None, quiet: bool = False) -> str | None:
    """Compile the reference shaders; returns the library path, or None when
    no reference checkout is present (the prebuilt library is then used)."""
    ref_root = ref_root or default_ref_root()
    if not os.path.isdir(os.path.join(ref_root, SHADER_DIR)):
        return OUT_LIB if os.path.exists(OUT_LIB) else None
    os.makedirs(OUT_DIR, exist_ok=True)
    tu = translation_unit(ref_root)
    for out, defs in ((OUT_LIB, []), (OUT_LIB_LIBM, ["-DRC_REF_HOST_LIBM"])):
        cmd = ["g++", "-std=c++20", "-O2", "-fopenmp", "-fwrapv", "-ffp-contract=off",
               "-fno-fast-math", "-fPIC", "-shared", "-w"] + defs + [
               "-I", HERE, "-I", os.path.join(REPO, "include"),
               "-x", "c++", "-", "-o", out + ".tmp"]
        proc = subprocess.run(cmd, input=tu.encode(), capture_output=True)
        if proc.returncode != 0:
            sys.stderr.write(proc.stderr.decode(errors="replace"))
            raise RuntimeError("building oracle/_ref failed")
        os.replace(out + ".tmp", out)
        if not quiet:
            print(f"built {out}")
    return OUT_LIB


if __name__ == "__main__":
    build(sys.argv[1] if len(sys.argv) > 1 else None)
