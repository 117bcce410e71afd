"""Build libhdgx.so (every CUDA source under hdg_b200/csrc) in-tree for sm_100a."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB = HERE / "libhdgx.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-I", str(HERE.parent / "include")]


# Per-file options.  elemental*.cu: device functions that are not inlined (the boundary-flux
# routine, called from the rarely taken boundary branch of the face loop) are compiled for at
# most 96 registers so that every elemental kernel instantiation (launch bounds of 96 to 255
# registers per thread) can call them; the kernels' own limits come from their launch bounds.
def file_flags(name):
    return ["-maxrregcount=96"] if name.startswith("elemental") else []


def sources():
    return sorted(CSRC.glob("*.cu"))


def needs_build():
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "hdgx.h"]
    return any(p.stat().st_mtime > t for p in deps)


def build(verbose=False, force=False, jobs=None):
    if not force and not needs_build():
        return LIB
    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    procs = []
    objs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        objs.append(obj)
        cmd = [NVCC, *FLAGS, *file_flags(src.name), "-dc", "-c", str(src), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    ok = True
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(out)
        ok &= p.returncode == 0
    if not ok:
        raise RuntimeError("nvcc failed")
    tmp = LIB.with_suffix(".so.tmp")
    subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(tmp),
                    *map(str, objs), "-lcudart"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force=True)
    print(LIB)
