"""Build recipe for the reference simulators used as a TEST ORACLE.

This script is test infrastructure.  It compiles the reference package's own
Cython sources (``src/cssm/*.pyx`` of ssm-simulators) where they lie, with
``cython`` + ``g++-13`` invoked directly -- the reference's setup.py is not run.
The outputs go to ``oracle/_ref/cssm/`` only (git-ignored; they travel to the
GPU host next to the other built shared objects).  Nothing in the product
imports them: only tests, the smoke check and the CPU-baseline leg of the
benchmark load ``oracle/_ref``.

Compiler flags mirror the reference build for Linux x86-64
(setup.py:244-330: ``-O3 -ffast-math -march=x86-64-v2 -funroll-loops
-fopenmp``), so the timed CPU baseline is the reference's own code at its own
optimisation level.  GSL is absent on this image, so the parallel path is
compiled with the header's stubs and ``check_parallel_request`` clamps
``n_threads`` to 1 (src/cssm/_openmp_status.pyx:228-242).

The reference sources are found through ``reference_root()``: the
directory named by the environment variable ``SSM_REFERENCE_ROOT``, else a
checkout named ``reference`` beside this repository's own directory.

Usage:  python oracle/build_ref.py [--reference-root DIR]
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import sysconfig
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT_PKG = HERE / "_ref" / "cssm"
BUILD = HERE / "_ref" / "_build"

# Modules on the simulated hot path (plus the two they import at module level).
MODULES = ["_utils", "_openmp_status", "ddm_models", "race_models", "levy_models", "lba_models",
           "ornstein_models"]

CXX_FLAGS = ["-O3", "-ffast-math", "-march=x86-64-v2", "-funroll-loops", "-fopenmp",
             "-fPIC", "-shared", "-DHAVE_OPENMP=1", "-w"]


def reference_root() -> Path | None:
    """The reference source tree (a directory holding ``src/cssm`` and
    ``ssms``): ``$SSM_REFERENCE_ROOT``, else ``../reference`` relative to the
    repository root; None when neither exists."""
    env = os.environ.get("SSM_REFERENCE_ROOT")
    cand = Path(env) if env else HERE.parent.parent / "reference"
    return cand if (cand / "src" / "cssm").is_dir() else None


def _find_cxx() -> str:
    for cand in ("g++-13", "g++"):
        p = shutil.which(cand)
        if p:
            return p
    raise RuntimeError("no C++ compiler found for the reference oracle build")


def build(reference_root: Path, force: bool = False) -> Path:
    src = reference_root / "src" / "cssm"
    if not src.is_dir():
        raise FileNotFoundError(f"reference sources not found under {src}")
    import numpy  # noqa: PLC0415  (build-time only)

    OUT_PKG.mkdir(parents=True, exist_ok=True)
    BUILD.mkdir(parents=True, exist_ok=True)
    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    cxx = _find_cxx()
    inc = ["-I" + numpy.get_include(), "-I" + sysconfig.get_paths()["include"], "-I" + str(src)]
    for mod in MODULES:
        target = OUT_PKG / (mod + suffix)
        pyx = src / (mod + ".pyx")
        if target.exists() and not force and target.stat().st_mtime > pyx.stat().st_mtime:
            continue
        cpp = BUILD / (mod + ".cpp")
        subprocess.check_call([sys.executable, "-m", "cython", "--cplus", "-3",
                               "-I", str(src), "--module-name", f"cssm.{mod}",
                               str(pyx), "-o", str(cpp)])
        subprocess.check_call([cxx, *CXX_FLAGS, *inc, str(cpp), "-o", str(target)])
        print(f"built {target.relative_to(HERE)}")
    # A package marker of our own: importing a module pulls in only what it needs.
    (OUT_PKG / "__init__.py").write_text(
        '"""Reference simulators compiled as a test oracle (see oracle/build_ref.py)."""\n')
    return OUT_PKG.parent


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference-root", default=None,
                    help="reference source tree (default: $SSM_REFERENCE_ROOT, else ../reference)")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    root = Path(args.reference_root) if args.reference_root else reference_root()
    if root is None:
        raise SystemExit("reference sources not found: set SSM_REFERENCE_ROOT or pass --reference-root")
    build(root, force=args.force)


if __name__ == "__main__":
    main()
