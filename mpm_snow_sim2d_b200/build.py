"""Build the solver's CUDA library in-tree for B200 (sm_100a).

``python -m mpm_snow_sim2d_b200.build`` compiles ``csrc/*.cu`` into
``mpm_snow_sim2d_b200/libmpm_b200.so`` with nvcc. The library exposes the
C ABI declared in ``include/mpm/mpm.h`` and nothing else.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libmpm_b200.so"

GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libmpm_b200.so")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the CUDA library if any source or header is newer than it."""
    deps = sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted((INCLUDE / "mpm").glob("*.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [
        nvcc_path(), *GENCODE, "-lineinfo", "-O3", "-std=c++17",
        "-Xcompiler", "-fPIC,-fvisibility=hidden", "-shared",
        "--expt-relaxed-constexpr", "-Xptxas", "-v" if verbose else "-O3",
        "-I", str(INCLUDE), "-I", str(CSRC),
        "-DMPM_BUILDING_LIBRARY",
        *[str(s) for s in sources()],
        "-o", str(tmp),
    ]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    if verbose:
        sys.stderr.write(res.stdout + res.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
