"""Builds the native parts in-tree.

  php_fdtd_b200/libphpfdtd.so   CUDA C ABI (include/php_fdtd.h), sm_100a
  php_fdtd_b200/libphphost.so   C host layer (include/php_host.h), no CUDA
  php_fdtd_b200/fdtd_b200       drop-in solver executable
  oracle/liboracle.so           CPU restatement (test infrastructure)
  oracle/_ref/*                 the reference solver and post-processor, when
                                PHP_REFERENCE_DIR names the reference checkout

Run ``python -m php_fdtd_b200.build`` or call ``build()``.  Each target is
rebuilt only when one of its inputs is newer.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
INC = ROOT / "include"
CSRC = PKG / "csrc"
HOST = PKG / "host"
ORACLE = ROOT / "oracle"

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _cc() -> str:
    return "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else (shutil.which("gcc") or "cc")


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def build_host(verbose: bool = False) -> Path:
    out = PKG / "libphphost.so"
    deps = [HOST / "php_host.c", INC / "php_host.h", INC / "php_fdtd.h", INC / "php_serve.h"]
    if _stale(out, deps):
        _run([_cc(), "-O2", "-ffp-contract=off", "-fno-fast-math", "-std=gnu11", "-fPIC", "-shared",
              "-Wall", "-Wextra", "-Wno-unused-parameter", "-Wno-format-truncation", f"-I{INC}", HOST / "php_host.c",
              "-lm", "-o", out], verbose)
    return out


def build_device(verbose: bool = False) -> Path:
    out = PKG / "libphpfdtd.so"
    sources = [CSRC / "php_fdtd.cu", CSRC / "php_noalloc.cu", CSRC / "php_serve.cu"]
    deps = sources + [INC / "php_fdtd.h", INC / "php_serve.h"] + [p for p in CSRC.glob("*.cuh")]
    if _stale(out, deps):
        _run([_nvcc(), *NVCC_ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-shared", f"-I{INC}", *sources, "-o", out], verbose)
    return out


def build_cli(verbose: bool = False) -> Path:
    out = PKG / "fdtd_b200"
    deps = [HOST / "fdtd_b200_main.c", INC / "php_host.h", INC / "php_fdtd.h", PKG / "libphphost.so", PKG / "libphpfdtd.so"]
    if _stale(out, deps):
        _run([_cc(), "-O2", "-std=gnu11", "-pthread", "-Wall", "-Wextra", "-Wno-unused-parameter", f"-I{INC}",
              HOST / "fdtd_b200_main.c", f"-L{PKG}", "-lphphost", "-lphpfdtd", "-Wl,-rpath,$ORIGIN", "-lm", "-o", out],
             verbose)
    return out


def reference_dir() -> Path | None:
    """The reference checkout named by PHP_REFERENCE_DIR, if it holds fdtd.c."""
    v = os.environ.get("PHP_REFERENCE_DIR", "")
    return Path(v) if v and (Path(v) / "fdtd.c").exists() else None


def build_oracle(verbose: bool = False) -> None:
    targets = ["restatement"]
    ref = reference_dir()
    if ref is not None:
        targets.append("ref")
    cmd = ["make", "-s", "-C", ORACLE, *([f"REF={ref}"] if ref is not None else []), *targets]
    _run(cmd, verbose)


def build(verbose: bool = False) -> None:
    build_host(verbose)
    build_device(verbose)
    build_cli(verbose)
    build_oracle(verbose)


if __name__ == "__main__":
    build(verbose="-q" not in sys.argv)
