"""Builds ``cubokit_b200/libcuboptycho.so`` from ``csrc/*.cu`` with nvcc for sm_100a (B200), in-tree.

Usage: ``python -m cubokit_b200.build`` (or ``build()`` from Python).  Rebuilds only when a source is newer than the
library.  ``ptxas_verbose=True`` prints register and shared-memory use of every kernel.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
LIB = HERE / "libcuboptycho.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(CSRC.glob("*.cu"))


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*")) + list(INCLUDE.glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr"]
OBJ = HERE / "_build"


def _compile(src: Path, ptxas_verbose: bool):
    obj = OBJ / (src.stem + ".o")
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))
    newest = max([src.stat().st_mtime] + [h.stat().st_mtime for h in headers])
    if obj.exists() and obj.stat().st_mtime > newest and not ptxas_verbose:
        return obj, ""
    cmd = [nvcc(), *ARCH, *FLAGS, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src), "-o", str(obj) + ".tmp"]
    if ptxas_verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}{res.stderr}")
    os.replace(str(obj) + ".tmp", obj)
    return obj, res.stderr


def build(force: bool = False, ptxas_verbose: bool = False, quiet: bool = False) -> Path:
    if not force and not stale() and not ptxas_verbose:
        return LIB
    OBJ.mkdir(exist_ok=True)
    if force:
        for o in OBJ.glob("*.o"):
            o.unlink()
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(sources()), os.cpu_count() or 1))) as pool:
        results = list(pool.map(lambda s: _compile(s, ptxas_verbose), sources()))
    if ptxas_verbose:
        for _, log in results:
            sys.stderr.write(log)
    cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB) + ".tmp", *[str(o) for o, _ in results], "-lcudart"]
    if not quiet:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc link failed")
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, ptxas_verbose="-v" in sys.argv)
    print(LIB)
