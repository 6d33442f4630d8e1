"""Build recipe of the native libraries (in-tree, so they travel with the repo).

  cuopus_b200/lib/libcuopus.so            the product: CUDA kernels for sm_100a
                                          plus the C ABI of include/cuopus.h
  cuopus_b200/lib/libcuopus_phases.so     the same with the decoder's stage timers
                                          (diagnostics: python bench.py --phases)
  cuopus_b200/lib/libcuopus_hostcheck.so  the same decoder sources compiled for
                                          the host (g++), used only by tests
  cuopus_b200/lib/libcuopus_lanesim.so    the host build with every lane of a
                                          group as a fiber, switched at random
                                          points (tests of the lane discipline)
  cuopus_b200/bin/cuopus_decode           the command-line tool / daemon

python -m cuopus_b200.build [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
BIN = os.path.join(HERE, "bin")
NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

LIBCUOPUS = os.path.join(LIB, "libcuopus.so")
LIBPHASES = os.path.join(LIB, "libcuopus_phases.so")
HOSTCHECK = os.path.join(LIB, "libcuopus_hostcheck.so")
HOSTCHECK_REV = os.path.join(LIB, "libcuopus_hostcheck_rev.so")
LANESIM = os.path.join(LIB, "libcuopus_lanesim.so")
CLI = os.path.join(BIN, "cuopus_decode")


def _sources(*names):
    out = []
    for n in names:
        p = os.path.join(CSRC, n)
        if os.path.isdir(p):
            out += [os.path.join(p, f) for f in sorted(os.listdir(p))]
        else:
            out.append(p)
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd):
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_libcuopus(force=False):
    deps = _sources("libcuopus.cu", "decode_kernel.cu", "costmodel.cu", "server.cu", "kernels.cuh", "ogg_demux.cpp",
                    "ogg_demux.h", "ordercost.cpp", "ordercost.h", "ordercost_coef.inc", "dec") + \
        [os.path.join(ROOT, "include", "cuopus.h")]
    if not force and not _stale(LIBCUOPUS, deps):
        return LIBCUOPUS
    os.makedirs(LIB, exist_ok=True)
    obj = os.path.join(LIB, "obj")
    os.makedirs(obj, exist_ok=True)
    common = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-I", CSRC]
    # The decoder kernel is built at NVVM -O1 and ptxas -O1 (decode_kernel.cu
    # explains): its machine code is a third smaller than at -O3, and under load
    # the kernel waits on instruction fetch, so the smaller code decodes faster;
    # the rest is -O3.
    _run(common + ["-Xcicc", "-O1", "-Xptxas", "-O1,-v", "-c", os.path.join(CSRC, "decode_kernel.cu"),
                   "-o", os.path.join(obj, "decode_kernel.o")])
    _run(common + ["-Xptxas", "-v", "-c", os.path.join(CSRC, "libcuopus.cu"), "-o", os.path.join(obj, "libcuopus.o")])
    _run(common + ["-Xptxas", "-v", "-c", os.path.join(CSRC, "costmodel.cu"), "-o", os.path.join(obj, "costmodel.o")])
    _run(common + ["-c", os.path.join(CSRC, "server.cu"), "-o", os.path.join(obj, "server.o")])
    _run(common + ["-c", os.path.join(CSRC, "ogg_demux.cpp"), "-o", os.path.join(obj, "ogg_demux.o")])
    _run(common + ["-c", os.path.join(CSRC, "ordercost.cpp"), "-o", os.path.join(obj, "ordercost.o")])
    tmp = LIBCUOPUS + ".tmp"
    rest = [os.path.join(obj, o) for o in ("libcuopus.o", "costmodel.o", "server.o", "ogg_demux.o", "ordercost.o")]
    _run([NVCC, *ARCH, "-shared", "-o", tmp, os.path.join(obj, "decode_kernel.o")] + rest)
    os.replace(tmp, LIBCUOPUS)
    # diagnostic build: the same library with the decoder's stage timers on
    _run(common + ["-Xcicc", "-O1", "-Xptxas", "-O1", "-DCUO_PHASE_TIMERS", "-c",
                   os.path.join(CSRC, "decode_kernel.cu"), "-o", os.path.join(obj, "decode_kernel_phases.o")])
    tmp = LIBPHASES + ".tmp"
    _run([NVCC, *ARCH, "-shared", "-o", tmp, os.path.join(obj, "decode_kernel_phases.o")] + rest)
    os.replace(tmp, LIBPHASES)
    return LIBCUOPUS


def build_hostcheck(force=False):
    """The host build, and a second one whose lane-split loops run backwards
    (a test that their iterations are independent)."""
    deps = _sources("hostcheck.cpp", "dec")
    for target, extra in ((HOSTCHECK, []), (HOSTCHECK_REV, ["-DCUO_LFOR_REVERSE"])):
        if not force and not _stale(target, deps):
            continue
        os.makedirs(LIB, exist_ok=True)
        tmp = target + ".tmp"
        _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-w", "-I", CSRC, *extra,
              os.path.join(CSRC, "hostcheck.cpp"), "-o", tmp, "-lpthread"])
        os.replace(tmp, target)
    # the lane-interleaving build (lanesim.cpp): each lane a fiber, switched
    # at function entries (-finstrument-functions; -Bsymbolic binds the entry
    # hook to the library's own, not libc's empty one)
    deps = _sources("lanesim.cpp", "dec")
    if force or _stale(LANESIM, deps):
        os.makedirs(LIB, exist_ok=True)
        tmp = LANESIM + ".tmp"
        _run(["g++", "-O1", "-g", "-fno-omit-frame-pointer", "-std=c++17", "-fPIC", "-shared", "-w", "-I", CSRC,
              "-DCUO_LANE_SIM", "-finstrument-functions", os.path.join(CSRC, "lanesim.cpp"), "-o", tmp,
              "-lpthread", "-ldl", "-Wl,-Bsymbolic"])
        os.replace(tmp, LANESIM)
    return HOSTCHECK


def build_cli(force=False):
    src = os.path.join(CSRC, "cli.cpp")
    if not os.path.exists(src):
        return None
    deps = [src, os.path.join(ROOT, "include", "cuopus.h"), LIBCUOPUS]
    if not force and not _stale(CLI, deps):
        return CLI
    os.makedirs(BIN, exist_ok=True)
    cuda = os.path.dirname(os.path.dirname(NVCC))
    _run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"),
          src, "-o", CLI + ".tmp", "-L", LIB, "-lcuopus", "-Wl,-rpath,$ORIGIN/../lib",
          "-L", os.path.join(cuda, "lib64"), "-lcudart_static", "-ldl", "-lrt", "-lpthread"])
    os.replace(CLI + ".tmp", CLI)
    return CLI


def build_all(force=False):
    build_libcuopus(force)
    build_hostcheck(force)
    build_cli(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
