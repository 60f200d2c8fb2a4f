"""Builds the native parts in-tree.

  fermiphasespace_b200/_lib/libfpsg.so   CUDA kernels + C ABI (sm_100a)
  fermiphasespace_b200/_lib/libfpshost.so, fps, makeSitesSystem   C++ host layer
  oracle/_build/liboracle.so             FP64 oracle (test infrastructure)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_DIR = os.path.join(HERE, "_lib")
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _sources(d: str, exts) -> list[str]:
    if not os.path.isdir(d):
        return []
    return sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith(exts))


def build_cuda(force: bool = False, verbose: bool = False) -> str:
    """Compiles the CUDA translation units in parallel, then links libfpsg.so."""
    os.makedirs(LIB_DIR, exist_ok=True)
    obj_dir = os.path.join(LIB_DIR, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    out = os.path.join(LIB_DIR, "libfpsg.so")
    headers = _sources(CSRC, (".cuh", ".h")) + [os.path.join(ROOT, "include", "fpsg.h")]
    units = _sources(CSRC, (".cu",))
    flags = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]
    if verbose:
        flags.append("-Xptxas=-v")
    procs, objs = [], []
    for u in units:
        o = os.path.join(obj_dir, os.path.basename(u)[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, [u] + headers):
            procs.append(subprocess.Popen([NVCC, *flags, "-c", "-o", o, u], cwd=ROOT))
    for pr in procs:
        if pr.wait() != 0:
            raise subprocess.CalledProcessError(pr.returncode, pr.args)
    if force or _stale(out, objs):
        subprocess.run([NVCC, *ARCH, "-shared", "-o", out, *objs], check=True, cwd=ROOT)
    return out


def build_host(force: bool = False) -> list[str]:
    """C++ host layer: JSON, lattice/system builders, solvers, fps CLI."""
    srcs = _sources(HOST, (".cpp",))
    if not srcs:
        return []
    hdrs = _sources(HOST, (".h", ".hpp")) + [os.path.join(ROOT, "include", "fpsg.h"),
                                               os.path.join(ROOT, "include", "fps_host.h")]
    lib_srcs = [s for s in srcs if not os.path.basename(s).startswith("main_")]
    outs = []
    lib = os.path.join(LIB_DIR, "libfpshost.so")
    flags = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wextra", f"-I{os.path.join(ROOT, 'include')}"]
    if force or _stale(lib, srcs + hdrs + [os.path.join(LIB_DIR, "libfpsg.so")]):
        subprocess.run([CXX, *flags, "-shared", "-o", lib, *lib_srcs, f"-L{LIB_DIR}", "-lfpsg",
                        "-Wl,-rpath,$ORIGIN"], check=True, cwd=ROOT)
    outs.append(lib)
    for m in [s for s in srcs if os.path.basename(s).startswith("main_")]:
        name = os.path.basename(m)[len("main_"):-len(".cpp")]
        exe = os.path.join(LIB_DIR, name)
        if force or _stale(exe, [m, lib]):
            subprocess.run([CXX, *flags, "-o", exe, m, f"-L{LIB_DIR}", "-lfpshost", "-lfpsg",
                            "-Wl,-rpath,$ORIGIN"], check=True, cwd=ROOT)
        outs.append(exe)
    return outs


def build_oracle() -> str:
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    return os.path.join(ROOT, "oracle", "_build", "liboracle.so")


def build_all(force: bool = False) -> None:
    build_cuda(force)
    build_host(force)
    build_oracle()


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
