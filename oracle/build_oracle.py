"""Build recipe for the oracle (test infrastructure only).

* ``oracle/liboracle_mpm.so`` — the project's CPU restatement (mpm_oracle.cpp),
  FP64 oracle + FP32/OpenMP CPU baseline.
* ``oracle/_ref/poisson{2,3}d`` — the reference's Poisson-disk samplers
  (src/shared/Shapes.h, included where it lies) behind a small driver.
* ``oracle/_ref/refcpu_driver`` — the reference's own CPU path: src/cpu/Grid.cpp
  and src/cpu/Particles.cpp compiled unmodified, where they lie in the reference
  tree, with g++ against the shadow headers in oracle/refcpu/shadow (runtime
  Parameters.h knobs, a project-written Eigen/Dense 2x2 stand-in because the
  vendored Eigen lacks Core, and the three helpers.h conversions). Built only
  when the reference tree is present; nothing is copied out of it and the
  binary stays in the git-ignored oracle/_ref/.
* ``oracle/_ref/libshader_ref.so`` — the reference's GPU path: its GLSL compute
  shaders (src/gpu/shaders/{2d,3d}) turned into C++ by oracle/shader/glsl_cpp.py
  (generated fragments in oracle/_ref/shader/) and run on the CPU by
  oracle/shader/shader_runner.cpp against the vendored glm 0.9.7.1.

The reference tree is found at $MPM_REFERENCE_ROOT, else as the directory
`reference` beside this repository's root.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_ROOT = Path(os.environ.get("MPM_REFERENCE_ROOT") or (HERE.parent.parent / "reference"))
ORACLE_LIB = HERE / "liboracle_mpm.so"
REF_DIR = HERE / "_ref"
REFCPU = REF_DIR / "refcpu_driver"
POISSON = {2: REF_DIR / "poisson2d", 3: REF_DIR / "poisson3d"}
SHADER_LIB = REF_DIR / "libshader_ref.so"


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(map(str, cmd)) + "\n" + res.stdout + res.stderr)


def build_oracle(force: bool = False) -> Path:
    src = HERE / "mpm_oracle.cpp"
    if force or _stale(ORACLE_LIB, [src]):
        tmp = ORACLE_LIB.with_suffix(".so.tmp")
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", str(src), "-o", str(tmp)])
        os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def reference_available() -> bool:
    return (REF_ROOT / "src" / "cpu" / "Particles.cpp").exists()


def build_refcpu(force: bool = False) -> Path | None:
    """Compile the reference CPU path; returns None when the reference tree is absent."""
    if not reference_available():
        return REFCPU if REFCPU.exists() else None
    shadow = HERE / "refcpu" / "shadow"
    driver = HERE / "refcpu" / "refcpu_driver.cpp"
    ref_srcs = [REF_ROOT / "src" / "cpu" / "Grid.cpp", REF_ROOT / "src" / "cpu" / "Particles.cpp"]
    deps = ref_srcs + [driver] + list(shadow.rglob("*"))
    if force or _stale(REFCPU, [d for d in deps if Path(d).is_file()]):
        REF_DIR.mkdir(exist_ok=True)
        tmp = REFCPU.with_suffix(".tmp")
        _run([
            "g++", "-O2", "-std=c++17", "-w",
            "-I", str(shadow),                       # shadow Parameters.h, helpers.h, Eigen/Dense first
            "-I", str(REF_ROOT / "src" / "shared"),  # Shapes.h
            "-I", str(REF_ROOT / "src" / "cpu"),
            "-I", str(REF_ROOT / "external" / "glm-0.9.7.1"),
            *map(str, ref_srcs), str(driver), "-o", str(tmp), "-pthread",
        ])
        os.replace(tmp, REFCPU)
    return REFCPU


def build_poisson(force: bool = False) -> dict:
    """The reference's Poisson-disk samplers (src/shared/Shapes.h) behind a
    small driver; {dim: path}, empty when the reference tree is absent."""
    if not reference_available():
        return {d: p for d, p in POISSON.items() if p.exists()}
    driver = HERE / "refcpu" / "poisson_driver.cpp"
    shapes = REF_ROOT / "src" / "shared" / "Shapes.h"
    for dim, out in POISSON.items():
        if force or _stale(out, [driver, shapes]):
            REF_DIR.mkdir(exist_ok=True)
            tmp = out.with_suffix(".tmp")
            _run(["g++", "-O2", "-std=c++17", "-w", *(["-DSIM_3D"] if dim == 3 else []),
                  "-I", str(REF_ROOT / "src" / "shared"), "-I", str(REF_ROOT / "external" / "glm-0.9.7.1"),
                  str(driver), "-o", str(tmp)])
            os.replace(tmp, out)
    return dict(POISSON)


def build_shader_ref(force: bool = False) -> Path | None:
    """The reference's GLSL step compiled for the CPU; None when neither the
    reference tree nor an earlier build is present."""
    shaders = REF_ROOT / "src" / "gpu" / "shaders"
    if not (shaders / "3d" / "p2g.glsl").exists():
        return SHADER_LIB if SHADER_LIB.exists() else None
    from .shader.glsl_cpp import generate
    gen_dir = REF_DIR / "shader"
    incs = generate(shaders, gen_dir)
    runner = HERE / "shader" / "shader_runner.cpp"
    if force or _stale(SHADER_LIB, incs + [runner, HERE / "shader" / "glsl_cpp.py"]):
        tmp = SHADER_LIB.with_suffix(".so.tmp")
        # GLSL reads unsuffixed floating literals as single precision
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-w", "-fsingle-precision-constant",
              "-I", str(gen_dir), "-I", str(REF_ROOT / "external" / "glm-0.9.7.1"), str(runner), "-o", str(tmp)])
        os.replace(tmp, SHADER_LIB)
    return SHADER_LIB


def build_all(force: bool = False) -> None:
    build_oracle(force)
    build_refcpu(force)
    build_poisson(force)
    build_shader_ref(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print(ORACLE_LIB, REFCPU if REFCPU.exists() else "(reference CPU path not built)")
