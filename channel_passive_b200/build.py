"""Build recipe for libkmm.so (sm_100a) and import check.

Compiles every CUDA / C++ source of channel_passive_b200/csrc with nvcc into one shared
library in channel_passive_b200/lib/, in tree, so that it travels with the repository.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libkmm.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = sources() + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "kmm.h"]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, extra=None) -> Path:
    if not force and not needs_build():
        return LIB
    LIBDIR.mkdir(exist_ok=True)
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    cc = nvcc()
    common = ["-O3", "-std=c++20", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I", str(PKG.parent / "include")] + ARCH + list(extra or [])
    objs = []
    procs = []
    for src in sources():
        obj = objdir / (src.name + ".o")
        cmd = [cc, "-c", str(src), "-o", str(obj)] + common
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    failed = False
    for cmd, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode:
            sys.stderr.write(" ".join(cmd) + "\n" + (out or ""))
        failed |= p.returncode != 0
    if failed:
        raise RuntimeError("libkmm compilation failed")
    tmp = LIBDIR / "libkmm.so.tmp"
    cmd = [cc, "-shared", "-o", str(tmp)] + [str(o) for o in objs] + ARCH + ["-lcudart_static"]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode:
        raise RuntimeError("libkmm link failed:\n" + r.stdout)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
