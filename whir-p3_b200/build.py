"""Build recipe for libwhir_b200.so (sm_100a) and, for tests, the oracle.

The CUDA sources are compiled in-tree with nvcc into whir-p3_b200/lib/ so the
library travels with the repository snapshot; no JIT cache is involved.
"""
from __future__ import annotations

import os
import pathlib
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libwhir_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources() -> list[pathlib.Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale(target: pathlib.Path, deps: list[pathlib.Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    deps = sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [PKG.parent / "include" / "whir_b200.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    LIB_DIR.mkdir(exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    cmds, objs = [], []
    for src in sources():
        obj = LIB_DIR / (src.stem + ".o")
        cmds.append([nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-c",
                     "-I", str(PKG.parent / "include"), str(src), "-o", str(obj)])
        objs.append(str(obj))
    # one nvcc per translation unit, in parallel
    import concurrent.futures

    def run(cmd):
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)

    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(run, c) for c in cmds]:
            f.result()
    cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
