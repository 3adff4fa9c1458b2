"""Build the in-tree native libraries.

* ``pelagos_b200/_lib/librelaybp.so``: the sm_100a kernels and the C ABI of
  include/relaybp.h, compiled by nvcc for ``-gencode arch=compute_100a,code=sm_100a``
  with ``--fmad=false`` (no implicit multiply-add contraction) and the CUDA
  runtime linked statically;
* ``oracle/_build/liboracle.so``: the CPU oracle (test infrastructure).

Usage: ``python -m pelagos_b200.build``.
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
OUT = PKG / "_lib" / "librelaybp.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _compile_cmd(src: Path, obj: Path) -> list[str]:
    return [nvcc(), *ARCH, "-lineinfo", "-O3", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
            "-Xcompiler", "-fvisibility=hidden", f"-I{ROOT / 'include'}", "-c", "-o", str(obj), str(src)]


def native_cmd(out: Path = OUT) -> list[str]:
    """Link step (after every source is compiled to an object next to `out`)."""
    objs = [str(out.parent / (s.stem + ".o")) for s in sources()]
    return [nvcc(), *ARCH, "-shared", "-cudart", "static", "-Xcompiler", "-fvisibility=hidden",
            "-o", str(out), *objs]


def build_native(force: bool = False, verbose: bool = True) -> Path:
    """Compile the sources in parallel (one nvcc per file), then link the shared library."""
    from concurrent.futures import ThreadPoolExecutor

    OUT.parent.mkdir(parents=True, exist_ok=True)
    deps = sources() + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "relaybp.h", Path(__file__)]
    if not force and OUT.exists() and all(OUT.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return OUT
    jobs = [(s, OUT.parent / (s.stem + ".o")) for s in sources()]

    def run(job):
        cmd = _compile_cmd(*job)
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(run, jobs))
    cmd = native_cmd()
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return OUT


def build_oracle(verbose: bool = True) -> Path:
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    return ROOT / "oracle" / "_build" / "liboracle.so"


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    build_native(force="--force" in argv)
    build_oracle()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
