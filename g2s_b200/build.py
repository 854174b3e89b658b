"""Build recipe for the CUDA extension (sm_100a) and the drop-in device.

    python -m g2s_b200.build          # -> g2s_b200/libg2s_b200.so
    python -m g2s_b200.build dropin   # -> g2s_b200/dropin/g2s_cuda.so (needs the G2S headers)
    python -m g2s_b200.build cli      # -> g2s_b200/qs_b200 (the G2S `qs` command line)

nvcc cross-compiles for sm_100a without a GPU.  The shared library is built
in-tree so that it travels with the repository to the GPU machine.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libg2s_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOSTCXX = "/usr/bin/g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["qsk_kernels.cu", "qsk_tc.cu", "qsk_peaks.cu", "qsk_learn.cu", "qsk_host.cpp", "qsk_tensor.cpp",
           "qsk_encoder.cpp", "qsk_bgrid.cpp"]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_lib(force: bool = False) -> str:
    deps = [os.path.join(CSRC, s) for s in SOURCES] + [os.path.join(CSRC, "qsk_internal.h"),
                                                       os.path.join(CSRC, "qsk_host_util.h"),
                                                       os.path.join(CSRC, "qsk_encoder.h"),
                                                       os.path.join(CSRC, "qsk_pdl.cuh"),
                                                       os.path.join(CSRC, "qsk_tc_nodes.cuh"),
                                                       os.path.join(ROOT, "include", "g2s_b200.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    objs = []
    for src in SOURCES:
        obj = os.path.join(CSRC, src.rsplit(".", 1)[0] + ".o")
        cmd = [NVCC, "-ccbin", HOSTCXX, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "-I", os.path.join(ROOT, "include"), "-c", os.path.join(CSRC, src), "-o", obj]
        if src.endswith(".cpp"):
            cmd[cmd.index("-c"):cmd.index("-c")] = ["-x", "cu"]
        _run(cmd)
        objs.append(obj)
    _run([NVCC, "-ccbin", HOSTCXX, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart", "-lz"])
    for o in objs:
        os.remove(o)
    return LIB


CLI = os.path.join(PKG, "qs_b200")


def build_cli() -> str:
    """qs_b200: the G2S `qs` command line on this library (host C++)."""
    build_lib()
    _run([HOSTCXX, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), os.path.join(PKG, "cli", "qs_b200.cpp"),
          "-o", CLI, "-L", PKG, "-lg2s_b200", "-Wl,-rpath,$ORIGIN"])
    # auto_qs_b200: the G2S `auto_qs` calibration command line
    _run([HOSTCXX, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
          os.path.join(PKG, "cli", "auto_qs_b200.cpp"), "-o", os.path.join(PKG, "auto_qs_b200"), "-L", PKG,
          "-lg2s_b200", "-Wl,-rpath,$ORIGIN"])
    return CLI


DROPIN = os.path.join(PKG, "dropin")


def g2s_sources() -> str:
    """The G2S source tree: $G2S_SOURCES, else a `reference` directory beside
    this repository (where it lies when the build runs next to it)."""
    return os.environ.get("G2S_SOURCES") or os.path.join(os.path.dirname(ROOT), "reference")


def build_dropin(g2s_tree: str = "") -> str:
    """g2s_cuda.so for G2S `qs -W_CUDA`: compiled with the G2S host compiler
    against the G2S headers (its AcceleratorDevice class), linked to
    libg2s_b200.so found next to it ($ORIGIN/..)."""
    build_lib()
    out = os.path.join(DROPIN, "g2s_cuda.so")
    inc = os.path.join(g2s_tree or g2s_sources(), "include")
    if not os.path.isdir(inc):
        raise FileNotFoundError(f"G2S headers not found under {inc}")
    _run([HOSTCXX, "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-w", "-DG2S_PATH_INDEX_TYPE=unsigned",
          "-I", inc, "-I", os.path.join(ROOT, "oracle", "fftw_shim"), "-I", os.path.join(ROOT, "oracle", "json_stub"),
          "-I", os.path.join(ROOT, "include"), os.path.join(DROPIN, "g2s_cuda_device.cpp"), "-o", out,
          "-L", PKG, "-lg2s_b200", "-Wl,-rpath,$ORIGIN/..:$ORIGIN"])
    return out


if __name__ == "__main__":
    if "dropin" in sys.argv:
        build_dropin(*[a for a in sys.argv[1:] if a.startswith("/")])
    elif "cli" in sys.argv:
        build_cli()
    else:
        build_lib(force="--force" in sys.argv)
