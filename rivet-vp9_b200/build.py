#!/usr/bin/env python3
"""Builds the decoder library in-tree: rivet-vp9_b200/_build/librv9.so.

The CUDA kernels are compiled for sm_100a (B200) only; the host parser, the
engine and the C ABI are compiled into the same shared library. nvcc
cross-compiles, so this runs on a machine without a GPU.

Usage: python rivet-vp9_b200/build.py [--force]
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "librv9.so")

SOURCES = [
    "gpu/kernels.cu",
    "gpu/parse_kernels.cu",
    "gpu/device_parse.cpp",
    "gpu/engine.cpp",
    "api/rv9_api.cpp",
    "serve/server.cpp",
    "serve/cluster.cpp",
    "host/parser.cpp",
    "host/probs.cpp",
]
HEADERS = [
    "api/api_internal.h",
    "gpu/dsp_math.cuh",
    "gpu/md5.cuh",
    "gpu/engine_types.h",
    "gpu/engine.h",
    "gpu/tile_parse.cuh",
    "gpu/parse_plan.h",
    "gpu/device_parse.h",
    "host/parser.h",
    "host/syntax.h",
    "host/probs.h",
    "host/bitreader.h",
    "common/vp9_tables.h",
    "common/vp9_consts.h",
]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# The host parser's token loop is a chain of dependent shifts and leading-zero
# counts: built for x86-64-v3 (BMI2 shifts, LZCNT) it runs about 5 % faster.
# The C ABI refuses to create a decoder or engine on a host CPU without it
# (rv9_api.cpp, built for the baseline ISA, checks before any parser code).
HOST_FLAGS = {"host/parser.cpp": ["-Xcompiler", "-march=x86-64-v3"]}


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    deps += [os.path.join(HERE, "..", "include", h) for h in ("rv9.h", "rv9_records.h", "rv9_server.h")]
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps)


ENC_LIB = os.path.join(OUT, "librv9enc.so")
ENC_SOURCES = ["encoder/encoder.cpp", "host/probs.cpp"]
ENC_HEADERS = ["encoder/recon_host.h", "host/syntax.h", "host/parser.h", "host/probs.h", "gpu/dsp_math.cuh",
               "common/vp9_tables.h", "common/vp9_consts.h"]


def build_encoder(force=False, verbose=False):
    """The stream generator (host CPU code): _build/librv9enc.so."""
    deps = [os.path.join(CSRC, s) for s in ENC_SOURCES + ENC_HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "rv9_encoder.h"))
    if not force and os.path.exists(ENC_LIB) and all(os.path.getmtime(d) <= os.path.getmtime(ENC_LIB) for d in deps):
        return ENC_LIB
    os.makedirs(OUT, exist_ok=True)
    tmp = ENC_LIB + ".tmp"
    cmd = ["g++", "-std=c++17", "-O3", "-fPIC", "-shared", "-o", tmp] + [os.path.join(CSRC, s) for s in ENC_SOURCES]
    cmd += ["-lpthread"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, ENC_LIB)
    return ENC_LIB


def build(force=False, verbose=False):
    if not force and not stale():
        return LIB
    os.makedirs(OUT, exist_ok=True)
    objs, cmds = [], []
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(OUT, os.path.basename(s) + ".o")
        cmd = [nvcc(), "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
               *ARCH, *HOST_FLAGS.get(s, []), "-c", src, "-o", obj]
        if s.endswith(".cpp"):
            cmd[1:1] = ["-x", "cu"] if s.startswith("gpu/") else []
        if "-Xptxas" in os.environ.get("RV9_NVCC_FLAGS", ""):
            cmd += os.environ["RV9_NVCC_FLAGS"].split()
        if verbose:
            print(" ".join(cmd))
        cmds.append(cmd)
        objs.append(obj)
    # The translation units compile independently, side by side.
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(cmds)) as ex:
        for f in [ex.submit(subprocess.run, c, check=True) for c in cmds]:
            f.result()
    tmp = LIB + ".tmp"
    subprocess.run([nvcc(), "-shared", *ARCH, "-o", tmp, *objs, "-lcudart", "-lpthread"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
    print(build_encoder(force="--force" in sys.argv, verbose=True))
