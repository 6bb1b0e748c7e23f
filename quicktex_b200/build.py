"""Build recipe for the in-tree native libraries of quicktex_b200.

Outputs (next to this file, so they travel with the source tree):

  libquicktex_cuda.so                       the C-ABI (include/quicktex_cuda.h) + sm_100a kernels
  _quicktex.cpython-<ver>-<plat>.so          the pybind11 module, linked against the above

Kernels are compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``),
with -lineinfo for profiling and -fmad=false (no float contraction, as the reference's
x86-64 build has none). nvcc cross-compiles, so this runs on a machine
without a GPU.

Usage:  python quicktex_b200/build.py [--force]

(Run it as a script: importing the package needs the extension this builds.)
"""

from __future__ import annotations

import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(ROOT, "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB = os.path.join(HERE, "libquicktex_cuda.so")
EXT = os.path.join(HERE, "_quicktex" + sysconfig.get_config_var("EXT_SUFFIX"))
BLOB = os.path.join(HERE, "data", "bc1_order_tables.bin")

KERNEL_SRCS = ["qt_kernels.cu", "qt_noalloc.cu", "qt_resize.cu"]
HOST_SRCS = ["qt_capi.cpp", "qt_batch.cpp", "qt_server.cpp"]
# every header a source may include: the kernels include qt_bc1_thread.cuh
HEADERS = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))) + \
    [os.path.join(INCLUDE, "quicktex_cuda.h"), os.path.abspath(__file__)]  # this recipe: its flags


def _newer(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")


def _blob_header() -> str:
    out = os.path.join(BUILD, "qt_order_blob.inc")
    if _newer(out, [BLOB]):
        return out
    data = open(BLOB, "rb").read()
    with open(out + ".tmp", "w") as f:
        f.write("// generated from quicktex_b200/data/bc1_order_tables.bin by quicktex_b200/build.py\n")
        f.write("static const unsigned char kOrderBlob[] = {\n")
        for i in range(0, len(data), 32):
            f.write(",".join(str(b) for b in data[i:i + 32]) + ",\n")
        f.write("};\nstatic const size_t kOrderBlobSize = %d;\n" % len(data))
    os.replace(out + ".tmp", out)
    return out


def build(force: bool = False, verbose: bool = False) -> None:
    os.makedirs(BUILD, exist_ok=True)
    blob = _blob_header()
    objs = []
    for src in KERNEL_SRCS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or not _newer(o, [s] + HEADERS):
            # -fmad=false: no float multiply-add contraction anywhere, the reference's x86-64 SSE
            # arithmetic (one rounding per operation) whether or not an expression is written with
            # explicit round-to-nearest intrinsics
            cmd = [NVCC, "-O3", "-std=c++17", *ARCH, "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-I" + INCLUDE,
                   "-I" + CSRC, "-c", s, "-o", o]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            _run(cmd)
        objs.append(o)
    for src in HOST_SRCS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        if force or not _newer(o, [s, blob] + HEADERS):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wextra", "-I" + INCLUDE,
                  "-I" + CSRC, "-I" + BUILD, "-I" + os.path.join(CUDA_HOME, "include"), "-c", s, "-o", o])
        objs.append(o)
    if force or not _newer(LIB, objs):
        _run([NVCC, "-shared", *ARCH, "-Xcompiler", "-fPIC", "-o", LIB, *objs, "-lpthread"])

    bind = os.path.join(CSRC, "bindings.cpp")
    if force or not _newer(EXT, [bind, LIB, os.path.join(INCLUDE, "quicktex_cuda.h")]):
        import pybind11

        _run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden", "-I" + INCLUDE,
              "-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"], bind, "-o", EXT,
              "-L" + HERE, "-lquicktex_cuda", "-Wl,-rpath,$ORIGIN"])


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print("built", LIB, EXT)
