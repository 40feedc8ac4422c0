"""Build the in-tree CUDA library `libflyb200.so` for sm_100a.

    python -m flyb200.build [--force]

Compiles every csrc/*.cu with nvcc into one shared library next to this file. --fmad=false keeps
each float multiply and add separately rounded, as the reference builds its kernels
(flyverse/cuda.py:51), so the fused LIF update and the optic update reproduce the reference's
float arithmetic; the kernels are memory-bound, so the lost contraction costs nothing measurable.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG.parent / "csrc"
INCLUDE = PKG.parent.parent / "include"
OUT = PKG / "libflyb200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC,-fvisibility=hidden", "-shared",
         "-Xptxas", "-warn-spills"]


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def stale() -> bool:
    if not OUT.exists():
        return True
    newest = max(p.stat().st_mtime for p in [*sources(), *CSRC.glob("*.cuh"), *INCLUDE.glob("*.h")])
    return OUT.stat().st_mtime < newest


def nvcc() -> str:
    found = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(found).exists():
        raise RuntimeError("nvcc not found: the flyb200 CUDA library cannot be built")
    return found


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not stale():
        return OUT
    tmp = OUT.with_name(f"libflyb200.{os.getpid()}.so")
    cmd = [nvcc(), *ARCH, *FLAGS, f"-I{INCLUDE}", *map(str, sources()), "-o", str(tmp)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    tmp.replace(OUT)
    return OUT


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args()
    print(build(args.force, args.verbose))


if __name__ == "__main__":
    main()
