"""Build the in-tree CUDA library ``dwba_b200/libdwba_b200.so`` for sm_100a.

Usage: ``python -m dwba_b200.build`` (or ``__graft_entry__.build()``). nvcc
cross-compiles without a GPU; the shared object is placed next to this file
so it travels with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libdwba_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build dwba_b200")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def build_hostpack(verbose: bool = False, force: bool = False) -> str:
    """The CPython extension ``_hostpack`` (csrc/hostpack.c: packing of a batch's waves on the host),
    built with the C compiler against this interpreter's headers, next to this file."""
    import sysconfig
    src = os.path.join(CSRC, "hostpack.c")
    out = os.path.join(HERE, "_hostpack" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so"))
    if not force and os.path.exists(out) and os.path.getmtime(src) <= os.path.getmtime(out):
        return out
    cc = os.environ.get("CC") or shutil.which("gcc") or shutil.which("cc")
    if not cc:
        raise RuntimeError("a C compiler is required to build dwba_b200._hostpack")
    cmd = [cc, "-O2", "-shared", "-fPIC", "-I", sysconfig.get_paths()["include"], src, "-o", out + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    res = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if res.returncode != 0:
        raise RuntimeError("hostpack build failed:\n" + res.stdout.decode(errors="replace"))
    os.replace(out + ".tmp", out)
    return out


def build(verbose: bool = False, force: bool = False) -> str:
    build_hostpack(verbose, force)
    srcs = sources()
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(HERE, "..", "include", "dwba_b200.h"))
    if not force and os.path.exists(LIB):
        t_lib = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t_lib for d in deps):
            return LIB
    nvcc = _nvcc()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in srcs:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off",
               "-Xptxas", "-O3", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT), src))
        objs.append(obj)
    for p, src in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{out.decode(errors='replace')}")
        if verbose and out:
            print(out.decode(errors="replace"))
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    res = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if res.returncode != 0:
        raise RuntimeError("link failed:\n" + res.stdout.decode(errors="replace"))
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
