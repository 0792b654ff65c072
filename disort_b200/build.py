"""Build the native libraries of disort_b200 in-tree.

    python -m disort_b200.build          # libdsp.so (sm_100a) + the Python host module
    python -m disort_b200.build --phase-clock   # tracing build of the flux path (lib/phase/)

libdsp.so is compiled with nvcc for sm_100a only (-gencode arch=compute_100a,
code=sm_100a); the host-side Python module (_disortpp) is compiled with g++
against pybind11 and links libdsp.so by rpath.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _deps(*exts: str) -> list[str]:
    out = [os.path.join(REPO, "include", "dsp.h")]
    for root, _, files in os.walk(CSRC):
        out += [os.path.join(root, f) for f in files if f.endswith(exts)]
    return out


LIBDSP_SOURCES = ("dsp_capi.cu", "dsp_general.cu", "dsp_noalloc.cu")


def build_libdsp(force: bool = False) -> str:
    """libdsp.so: each translation unit compiled to an object in parallel, then linked."""
    os.makedirs(LIB, exist_ok=True)
    target = os.path.join(LIB, "libdsp.so")
    if not (force or _stale(target, _deps(".cu", ".cuh", ".h", ".hpp"))):
        return target
    objdir = os.path.join(LIB, "obj")
    os.makedirs(objdir, exist_ok=True)
    procs, objs = [], []
    for src in LIBDSP_SOURCES:
        obj = os.path.join(objdir, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-diag-suppress", "177",
               "-c", "-o", obj, os.path.join(CSRC, src)]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for cmd, pr in procs:
        outp, _ = pr.communicate()
        if pr.returncode != 0:
            failed.append(" ".join(cmd) + "\n" + outp)
    if failed:
        raise RuntimeError("nvcc failed:\n" + "\n".join(failed))
    _run([NVCC, *ARCH, "-shared", "-o", target, *objs])
    return target


def build_emu(force: bool = False) -> str:
    """libdsp_emu.so: the emulator's tcgen05 GEMMs, training loop and gate."""
    os.makedirs(LIB, exist_ok=True)
    target = os.path.join(LIB, "libdsp_emu.so")
    deps = [os.path.join(REPO, "include", "dsp_emu.h"), os.path.join(REPO, "include", "dsp.h")]
    deps += [os.path.join(CSRC, "emu", f) for f in os.listdir(os.path.join(CSRC, "emu"))]
    if force or _stale(target, deps):
        _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
              "-o", target, os.path.join(CSRC, "emu", "emu.cu")])
    return target


def build_bench(force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    target = os.path.join(LIB, "libdsp_bench.so")
    src = os.path.join(CSRC, "fp64_peak.cu")
    if force or _stale(target, [src, os.path.join(CSRC, "dsp_device.cuh")]):
        _run([NVCC, *ARCH, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-o", target, src])
    return target


CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def build_host(force: bool = False) -> str:
    """libdisortpp.so (the DisORT++ C++ API over the C ABI) and the _disortpp module."""
    host = os.path.join(CSRC, "host")
    inc = os.path.join(REPO, "include")
    lib = os.path.join(LIB, "libdisortpp.so")
    srcs = [os.path.join(host, "disortpp_flux.cpp"), os.path.join(host, "disortpp_general.cpp")]
    deps = srcs + [os.path.join(host, "phase_tables.inc"), os.path.join(inc, "disortpp", "disortpp.hpp"),
                   os.path.join(inc, "dsp.h"), os.path.join(LIB, "libdsp.so")]
    if force or _stale(lib, deps):
        _run([CXX, "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall", "-o", lib, *srcs,
              "-L" + LIB, "-ldsp", "-Wl,-rpath,$ORIGIN"])
    import pybind11
    ext = sysconfig.get_config_var("EXT_SUFFIX")
    mod = os.path.join(HERE, "_disortpp" + ext)
    src = os.path.join(host, "pybind_module.cpp")
    if force or _stale(mod, [src, lib, os.path.join(inc, "disortpp", "disortpp.hpp")]):
        _run([CXX, "-std=c++17", "-O2", "-fPIC", "-shared", "-fvisibility=hidden",
              "-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"],
              "-o", mod, src, "-L" + LIB, "-ldisortpp", "-ldsp", "-Wl,-rpath,$ORIGIN/lib"])
    return mod


def build_phase_clock(force: bool = False) -> str:
    """lib/phase/libdsp.so: libdsp.so with the flux path's phase markers counting
    cycles (csrc/instrument/phase_clock.cuh force-included into dsp_capi.cu);
    the other objects are the product build's.  Read by disort_b200.phase_profile."""
    target_dir = os.path.join(LIB, "phase")
    os.makedirs(target_dir, exist_ok=True)
    target = os.path.join(target_dir, "libdsp.so")
    build_libdsp()
    hdr = os.path.join(CSRC, "instrument", "phase_clock.cuh")
    if force or _stale(target, _deps(".cu", ".cuh", ".h", ".hpp") + [hdr]):
        obj = os.path.join(target_dir, "dsp_capi.o")
        _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-diag-suppress", "177",
              "-include", hdr, "-c", "-o", obj, os.path.join(CSRC, "dsp_capi.cu")])
        _run([NVCC, *ARCH, "-shared", "-o", target, obj, os.path.join(LIB, "obj", "dsp_general.o"),
              os.path.join(LIB, "obj", "dsp_noalloc.o")])
    return target


def build_all(force: bool = False) -> None:
    build_libdsp(force)
    build_emu(force)
    build_bench(force)
    build_host(force)


if __name__ == "__main__":
    if "--phase-clock" in sys.argv:
        build_phase_clock(force="--force" in sys.argv)
    else:
        build_all(force="--force" in sys.argv)
