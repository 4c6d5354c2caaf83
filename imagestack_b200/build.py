"""Build the CUDA library (and, where the reference sources are present, the ImageStack
plugin) in-tree.

    python -m imagestack_b200.build            # libpermgpu.so (+ plugin if possible)

Every kernel is compiled for sm_100a only.  lattice_d.cu is compiled once per number of
position dimensions (1..16) in parallel; the objects go to imagestack_b200/_build/ and
the shared library to imagestack_b200/libpermgpu.so.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libpermgpu.so")
PLUGIN = os.path.join(PKG, "libpermgpu_imagestack.so")
INCLUDE = os.path.join(ROOT, "include")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOSTCXX = "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
                  "-ccbin", HOSTCXX, "-I", CSRC, "-I", INCLUDE]
MAX_D = 16


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(INCLUDE, "permgpu.h"))
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def compile_units():
    os.makedirs(BUILD, exist_ok=True)
    hdrs = _headers()
    jobs = []
    for d in range(1, MAX_D + 1):
        src = os.path.join(CSRC, "lattice_d.cu")
        obj = os.path.join(BUILD, "lattice_d%d.o" % d)
        jobs.append((obj, [src] + hdrs, [NVCC] + NVFLAGS + ["-DPGPU_D=%d" % d, "-c", src, "-o", obj]))
    for name in sorted(os.listdir(CSRC)):
        if not name.endswith(".cu") or name == "lattice_d.cu":
            continue
        src = os.path.join(CSRC, name)
        obj = os.path.join(BUILD, name[:-3] + ".o")
        jobs.append((obj, [src] + hdrs, [NVCC] + NVFLAGS + ["-c", src, "-o", obj]))
    todo = [j for j in jobs if _stale(j[0], j[1])]
    if todo:
        with ThreadPoolExecutor(max_workers=max(2, os.cpu_count() or 4)) as ex:
            list(ex.map(lambda j: _run(j[2]), todo))
    return [j[0] for j in jobs]


def link(objs):
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-Xlinker", "--no-undefined"])
    return LIB


def reference_src():
    """The reference's src/ folder, for the plugin's headers: $IMAGESTACK_SRC if set, else
    whatever the oracle's Makefile (the recipe that reads the reference sources) reports;
    None where the sources are absent."""
    env = os.environ.get("IMAGESTACK_SRC")
    if env:
        return env if os.path.isdir(env) else None
    try:
        r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "print-src"],
                           capture_output=True, text=True, timeout=60)
    except (OSError, subprocess.SubprocessError):
        return None
    out = r.stdout.strip().splitlines()
    return out[-1] if r.returncode == 0 and out and os.path.isdir(out[-1]) else None


def build_plugin(ref_src=None):
    """ImageStack plugin: subclasses of the reference's Operation classes, so it compiles
    against the reference headers; built only where those headers exist."""
    src = os.path.join(CSRC, "plugin", "imagestack_plugin.cpp")
    REF_SRC = ref_src or reference_src()
    if not (REF_SRC and os.path.exists(src)):
        return None
    if _stale(PLUGIN, [src, LIB, os.path.join(INCLUDE, "permgpu.h")]):
        _run([HOSTCXX, "-std=gnu++0x", "-O2", "-fPIC", "-shared", "-w",
              "-DNO_SDL", "-DNO_JPEG", "-DNO_TIFF", "-DNO_PNG", "-DNO_FFTW", "-DNO_OPENEXR",
              "-I", REF_SRC, "-I", INCLUDE, "-include", os.path.join(REF_SRC, "main.h"),
              src, "-o", PLUGIN, "-L", PKG, "-lpermgpu", "-Wl,-rpath,$ORIGIN"])
    return PLUGIN


def build(plugin: bool = True):
    objs = compile_units()
    lib = link(objs)
    if plugin:
        build_plugin()
    return lib


if __name__ == "__main__":
    print(build(plugin="--no-plugin" not in sys.argv))
