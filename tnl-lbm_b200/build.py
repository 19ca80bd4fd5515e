"""Build the sm_100a shared library libtnl_lbm_b200.so in-tree.

    python tnl-lbm_b200/build.py [--force]

Compiles every csrc/*.cu with nvcc for sm_100a (-gencode
arch=compute_100a,code=sm_100a -lineinfo -O3) in parallel and links
lib/libtnl_lbm_b200.so.  Objects are rebuilt when their source, any header in
csrc/ or include/, or this script is newer than the object.  The collision
plugins of plugins/*.cu (csrc/plugin.cuh) are compiled in the same pass into
lib/plugins/<name>.so; build_plugin() compiles a user's plugin the same way.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libtnl_lbm_b200.so")
PLUGINS = os.path.join(PKG, "plugins")
PLUGIN_LIBDIR = os.path.join(LIBDIR, "plugins")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "-I" + os.path.join(ROOT, "include"), "-ccbin", "g++"]


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h")) + [os.path.abspath(__file__)]
    hdr_time = _newest(headers)
    jobs = []
    for src in sources:
        obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr_time):
            jobs.append((src, [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]))
    lib_jobs = len(jobs)
    os.makedirs(PLUGIN_LIBDIR, exist_ok=True)
    for src in sorted(glob.glob(os.path.join(PLUGINS, "*.cu"))):
        so = os.path.join(PLUGIN_LIBDIR, os.path.basename(src)[:-3] + ".so")
        if force or not os.path.exists(so) or os.path.getmtime(so) < max(os.path.getmtime(src), hdr_time):
            jobs.append((src, plugin_command(src, so)))

    def compile_one(job):
        src, cmd = job
        return src, subprocess.run(cmd, capture_output=True, text=True)

    failed = []
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            for src, r in ex.map(compile_one, jobs):
                if verbose or r.returncode != 0:
                    sys.stderr.write(r.stdout + r.stderr)
                if r.returncode != 0:
                    failed.append(src)
    if failed:
        raise RuntimeError("nvcc failed for: " + ", ".join(os.path.basename(f) for f in failed))
    jobs = jobs[:lib_jobs]
    objs = [os.path.join(OBJ, os.path.basename(s)[:-3] + ".o") for s in sources]
    if force or jobs or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    build_examples(force)
    return LIB


def plugin_command(src: str, out: str) -> list:
    """nvcc command that compiles the collision plugin source `src` (a .cu
    file using LBM_COLLISION_PLUGIN of csrc/plugin.cuh) into the shared
    library `out`: the library's own flags, only the launchers exported."""
    return [NVCC, *ARCH, *FLAGS, "-I" + CSRC, "-shared", "-o", out, src]


def build_plugin(src: str, out: str, verbose: bool = False) -> str:
    """Compile a user's collision plugin; returns the path of the .so."""
    os.makedirs(os.path.dirname(os.path.abspath(out)), exist_ok=True)
    r = subprocess.run(plugin_command(src, out), capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for plugin " + src)
    return out


def build_examples(force: bool = False) -> list:
    """C++ host programs over the C-ABI (tnl-lbm_b200/host/examples), built
    with g++ against lib/libtnl_lbm_b200.so."""
    out = []
    host = os.path.join(PKG, "host")
    for src in sorted(glob.glob(os.path.join(host, "examples", "*.cpp"))):
        exe = os.path.join(LIBDIR, os.path.basename(src)[:-4])
        deps = [src, os.path.join(host, "lbm_b200.hpp"), os.path.join(ROOT, "include", "tnl_lbm_b200.h"), LIB]
        if force or not os.path.exists(exe) or os.path.getmtime(exe) < _newest(deps):
            cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"), "-I" + host, src,
                   "-L" + LIBDIR, "-ltnl_lbm_b200", "-Wl,-rpath,$ORIGIN", "-o", exe]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("host example build failed:\n" + r.stdout + r.stderr)
        out.append(exe)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
