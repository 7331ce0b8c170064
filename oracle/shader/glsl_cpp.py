"""TEST INFRASTRUCTURE — the reference's GLSL compute shaders as C++.

Only the oracle build (oracle/build_oracle.py) uses this module. The reference's
GPU path is four GLSL compute shaders per dimension
(src/gpu/shaders/{2d,3d}/{reset,p2g,grid_update,g2p}.glsl, with common.glsl
spliced in where a shader says "// #include common.glsl", as
src/gpu/GPUSolver.cpp:298-378 does). There is no OpenGL stack here, but GLSL
compute code is near-C and the reference vendors glm 0.9.7.1, a C++ library
built to mirror GLSL's types and functions. This module turns each shader's
text into a C++ translation-unit fragment that compiles against glm, without
touching any arithmetic:

* `#version`, `#extension` and `layout(local_size_x = ...) in;` lines are
  dropped; `// #include common.glsl` is replaced by the converted common.glsl;
* a storage buffer `layout(std430, ...) buffer B { T name[]; };` becomes a
  pointer `static T* name` that the runner points at its arrays, and a
  `uniform T name;` a `static T name` that the runner sets;
* `out` / `inout` parameters become C++ references;
* the GLSL array constructor `T[n](a, b, ...)` becomes a brace list;
* the `.xyz` swizzle of a vec4 becomes glm's vec3(vec4) conversion;
* `void main()` becomes `void shader_main()` (each shader is compiled in a
  namespace of its own by oracle/shader/shader_runner.cpp).

GLSL's unsuffixed floating literals are single precision; the runner is
compiled with g++'s -fsingle-precision-constant so that C++ reads them the same
way. The generated fragments are written to the git-ignored oracle/_ref/shader/
when the reference tree is present; nothing of the reference is committed.
"""
from __future__ import annotations

import re
from pathlib import Path

STAGES = ("reset", "p2g", "grid_update", "g2p")

_BUFFER = re.compile(
    r"layout\s*\(\s*std430\s*,\s*binding\s*=\s*\d+\s*\)\s*(?:(?:readonly|writeonly|coherent|restrict|volatile)\s+)*"
    r"buffer\s+\w+\s*\{\s*(\w+)\s+(\w+)\s*\[\s*\]\s*;\s*\}\s*;")
_UNIFORM = re.compile(r"^(\s*)uniform\s+(\w+)\s+(\w+)\s*;", re.M)
_FUNC_SIG = re.compile(r"^(\s*(?:void|float|int|vec[234]|mat[234])\s+\w+\s*)\(([^)]*)\)", re.M)
_OUT_PARAM = re.compile(r"\b(?:out|inout)\s+(\w+)\s+(\w+)")
_ARRAY_CTOR = re.compile(r"=\s*\w+\s*\[\s*\d+\s*\]\s*\(")
_SWIZZLE_XYZ = re.compile(r"(\b\w+(?:\[[^\]\[]+\])?)\.xyz\b")
_MAIN = re.compile(r"\bvoid\s+main\s*\(\s*\)")
_DROP = re.compile(r"^\s*(#version|#extension|layout\s*\(\s*local_size_x).*$", re.M)


def _array_ctors(src: str) -> str:
    out, pos = [], 0
    for m in _ARRAY_CTOR.finditer(src):
        if m.start() < pos:
            continue
        # m.end() - 1 is the opening parenthesis; find its match
        depth, i = 0, m.end() - 1
        while True:
            c = src[i]
            depth += c == "("
            depth -= c == ")"
            if depth == 0:
                break
            i += 1
        out.append(src[pos:m.start()])
        out.append("= {" + src[m.end():i] + "}")
        pos = i + 1
    out.append(src[pos:])
    return "".join(out)


def _params(src: str) -> str:
    return _FUNC_SIG.sub(lambda m: m.group(1) + "(" + _OUT_PARAM.sub(r"\1& \2", m.group(2)) + ")", src)


def convert(src: str, common: str | None = None) -> str:
    """C++ text of one GLSL compute shader (or of common.glsl when common is None
    and the text has no main)."""
    s = _DROP.sub("", src)
    if common is not None:
        s = s.replace("// #include common.glsl", convert(common))
    s = _BUFFER.sub(lambda m: f"static {m.group(1)}* {m.group(2)} = nullptr;", s)
    s = _UNIFORM.sub(r"\1static \2 \3;", s)
    s = _params(s)
    s = _array_ctors(s)
    s = _SWIZZLE_XYZ.sub(r"vec3(\1)", s)
    s = _MAIN.sub("void shader_main()", s)
    return s


def generate(shader_root: Path, out_dir: Path) -> list[Path]:
    """Write {2d,3d}_{stage}.inc for every stage; returns the written paths."""
    out_dir.mkdir(parents=True, exist_ok=True)
    written = []
    for dim in ("2d", "3d"):
        common = (shader_root / dim / "common.glsl").read_text()
        for stage in STAGES:
            src = (shader_root / dim / f"{stage}.glsl").read_text()
            text = convert(src, common if "// #include common.glsl" in src else None)
            path = out_dir / f"{dim}_{stage}.inc"
            header = f"// generated from {dim}/{stage}.glsl by oracle/shader/glsl_cpp.py (do not edit)\n"
            if not path.exists() or path.read_text() != header + text:
                path.write_text(header + text)
            written.append(path)
    return written
