"""Build the in-tree native libraries.

* ``quantkos_b200/libquantkos_b200.so`` — the CUDA engine and its C ABI, compiled
  for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``), plus the
  ``quantkos`` command-line driver next to it.
* ``oracle/libqkoracle.so`` — the CPU restatement used as the parity oracle by the
  tests (test infrastructure; never loaded by the engine).
* ``oracle/_ref/libqkref{64,32}.so`` — the reference's own headers compiled against
  the host shim, only when the reference checkout is present.

Run ``python -m quantkos_b200.build``.  Objects go to ``quantkos_b200/_build/``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libquantkos_b200.so"
CLI = PKG / "quantkos"
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "libqkoracle.so"
REF_DIR = ORACLE_DIR / "ref_harness"
# Where the reference checkout lies: QK_REFERENCE_ROOT, else the build machine's checkout.
# This build recipe is the only place that names that location; the harness Makefile and
# the golden-fixture generator take it from here.
REFERENCE_ROOT = Path(os.environ.get("QK_REFERENCE_ROOT", "/root/reference"))

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++20", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
                     "-Xptxas", "-O3", "--expt-relaxed-constexpr"]
SOURCES = ["qk_paths.cu", "qk_lsm.cu", "qk_api.cu", "qk_serve.cu", "qk_config.cu", "qk_tune.cu", "qk_noalloc.cu"]


def _run(cmd: list[str], cwd: Path | None = None) -> None:
    proc = subprocess.run(cmd, cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"command failed ({proc.returncode}): {' '.join(cmd)}\n{proc.stdout}")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def build_engine(force: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "quantkos_b200.h"]
    srcs = [s for s in SOURCES if (CSRC / s).exists()]
    jobs = []
    for s in srcs:
        o = OBJ / (Path(s).stem + ".o")
        if force or _stale(o, [CSRC / s] + headers):
            jobs.append([NVCC, *NVCC_FLAGS, "-c", str(CSRC / s), "-o", str(o)])
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            list(ex.map(_run, jobs))
    objs = [OBJ / (Path(s).stem + ".o") for s in srcs]
    if force or _stale(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lpthread"])
    cli_src = CSRC / "qk_cli.cpp"
    if cli_src.exists() and (force or _stale(CLI, [cli_src, LIB])):
        _run(["g++", "-std=c++20", "-O2", "-o", str(CLI), str(cli_src), f"-I{ROOT / 'include'}",
              f"-L{PKG}", "-lquantkos_b200", f"-Wl,-rpath,$ORIGIN"])
    return LIB


def build_oracle(force: bool = False) -> Path:
    src = ORACLE_DIR / "qk_oracle.c"
    if force or _stale(ORACLE_LIB, [src, ROOT / "include" / "quantkos_b200.h"]):
        _run(["gcc", "-std=c11", "-O2", "-fPIC", "-shared", "-fopenmp", "-o", str(ORACLE_LIB), str(src), "-lm"])
    return ORACLE_LIB


def build_reference_oracle() -> bool:
    """Compile the reference headers against the host shim (needs the reference tree)."""
    if not (REFERENCE_ROOT / "include" / "core").is_dir():
        return False
    _run(["make", "-s", "-C", str(REF_DIR), f"REF_ROOT={REFERENCE_ROOT}"])
    return True


def main(argv: list[str]) -> int:
    force = "--force" in argv
    build_engine(force)
    build_oracle(force)
    if "--no-ref" not in argv:
        build_reference_oracle()
    print(f"built {LIB}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
