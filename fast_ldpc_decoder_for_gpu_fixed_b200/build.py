"""Builds the native library in-tree: libldpc_b200.so (sm_100a) and the C++ tools.

    python -m fast_ldpc_decoder_for_gpu_fixed_b200.build [--force]

nvcc cross-compiles for sm_100a without a GPU.  The outputs stay inside the
package directory so they travel with the source tree.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
CPP = os.path.join(HERE, "cpp")
LIB = os.path.join(HERE, "libldpc_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "nvcc")


def _sources(d, exts):
    return sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith(exts)) if os.path.isdir(d) else []


def _stale(target, deps):
    return not os.path.exists(target) or any(os.path.getmtime(p) > os.path.getmtime(target) for p in deps)


def _local_deps(path, seen=None):
    """The file and every local header it includes (#include "..."), recursively."""
    import re
    seen = set() if seen is None else seen
    path = os.path.normpath(path)
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path) as f:
        for inc in re.findall(r'^\s*#\s*include\s+"([^"]+)"', f.read(), re.M):
            _local_deps(os.path.join(os.path.dirname(path), inc), seen)
    return seen


def build_lib(force=False, verbose=False):
    """Compiles every csrc/*.cu to an object (in parallel), then links the shared library.
    A unit is recompiled when it or a local header it includes is newer than its object."""
    units = _sources(CSRC, (".cu",))
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    base = [NVCC, "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", *ARCH,
            "-I", os.path.join(ROOT, "include")]
    if verbose:
        base.append("-Xptxas=-v")
    procs, objs = [], []
    for u in units:
        obj = os.path.join(objdir, os.path.basename(u)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, sorted(_local_deps(u))):
            procs.append((u, subprocess.Popen(base + ["-c", "-o", obj, u])))
    for u, p in procs:
        if p.wait() != 0:
            raise RuntimeError("nvcc failed on %s" % u)
    if procs or _stale(LIB, objs):
        subprocess.check_call([NVCC, "-shared", *ARCH, "-o", LIB] + objs)
    return LIB


def build_tools(force=False):
    """C++ reference-compatible plugin classes and the main.cpp-style driver."""
    srcs = _sources(CPP, (".cpp", ".h", ".cu"))
    if not srcs:
        return None
    exe = os.path.join(CPP, "ldpc_sim")
    if force or _stale(exe, srcs + [LIB]):
        cmd = [NVCC, "-O2", "-std=c++17", *ARCH, "-I", os.path.join(ROOT, "include"), "-I", CPP,
               "-o", exe] + [s for s in srcs if s.endswith((".cpp", ".cu"))] + \
              ["-L", HERE, "-lldpc_b200", "-Xlinker", "-rpath=$ORIGIN/.."]
        subprocess.check_call(cmd)
    return exe


def build(force=False, verbose=False):
    lib = build_lib(force, verbose)
    build_tools(force)
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
