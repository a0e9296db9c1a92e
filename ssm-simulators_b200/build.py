"""Build the sm_100a shared library ``libssm_b200.so`` in-tree.

Every ``csrc/*.cu`` file is compiled for ``sm_100a`` only and linked into one
shared object placed next to the Python package (``ssms_b200/_lib/``), so the
built library travels with the source tree.  The CUDA runtime is linked
statically; streams created by PyTorch are driver objects and are shared.

Usage:  python ssm-simulators_b200/build.py [--force] [--verbose-ptxas]
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
from pathlib import Path

ROOT = Path(__file__).resolve().parent
CSRC = ROOT / "csrc"
INCLUDE = ROOT.parent / "include"
OBJ = ROOT / "_build"
OUT = ROOT / "ssms_b200" / "_lib" / "libssm_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xcompiler", "-O2"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libssm_b200.so")
    return cand


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def build(force: bool = False, verbose_ptxas: bool = False, jobs: int | None = None) -> Path:
    nvcc = _nvcc()
    OBJ.mkdir(parents=True, exist_ok=True)
    OUT.parent.mkdir(parents=True, exist_ok=True)
    hdr_mtime = max((h.stat().st_mtime for h in _headers()), default=0.0)
    objs: list[Path] = []
    procs: list[tuple[subprocess.Popen, Path]] = []
    for src in _sources():
        obj = OBJ / (src.stem + ".o")
        objs.append(obj)
        if (not force and obj.exists() and obj.stat().st_mtime > src.stat().st_mtime
                and obj.stat().st_mtime > hdr_mtime):
            continue
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src), "-o", str(obj)]
        if verbose_ptxas:
            cmd[1:1] = ["-Xptxas", "-v"]
        procs.append((subprocess.Popen(cmd), src))
        if len(procs) >= (jobs or os.cpu_count() or 4):
            p, s = procs.pop(0)
            if p.wait() != 0:
                raise RuntimeError(f"nvcc failed on {s}")
    for p, s in procs:
        if p.wait() != 0:
            raise RuntimeError(f"nvcc failed on {s}")
    lib_mtime = OUT.stat().st_mtime if OUT.exists() else 0.0
    if force or not OUT.exists() or any(o.stat().st_mtime > lib_mtime for o in objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", str(OUT), *map(str, objs), "-cudart", "static"]
        subprocess.check_call(cmd)
    return OUT


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    args = ap.parse_args()
    print(build(force=args.force, verbose_ptxas=args.verbose_ptxas))


if __name__ == "__main__":
    main()
