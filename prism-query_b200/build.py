"""Builds libprism_gpu.so (sm_100a) in-tree: prism-query_b200/prism_gpu/libprism_gpu.so.

nvcc cross-compiles without a GPU; object files go to prism-query_b200/_build/.
Usage: python prism-query_b200/build.py [--force] [--debug]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "prism_gpu", "libprism_gpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: Float64 arithmetic rounds after every operation (no FMA
# contraction), as the reference computes it
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "--fmad=false",
         "-I", INCLUDE, "-I", CSRC]
# device headers embedded into the library for run-time compiled kernels
JIT_HEADERS = ["common.cuh", "eval.cuh", "join_device.cuh", "agg_device.cuh"]


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return max(os.path.getmtime(h) for h in hs)


def compile_one(src: str, force: bool, extra) -> str:
    obj = os.path.join(BUILD, src[:-3] + ".o")
    s = os.path.join(CSRC, src)
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(s), headers_mtime()):
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", s, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def jit_headers_object(force: bool) -> str:
    """Embeds JIT_HEADERS as C strings (kJitHeaderNames / kJitHeaderTexts)."""
    src = os.path.join(BUILD, "jit_headers.cpp")
    obj = os.path.join(BUILD, "jit_headers.o")
    hs = [os.path.join(CSRC, h) for h in JIT_HEADERS]
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(h) for h in hs):
        return obj
    delim = "PRISMHDR"
    parts = []
    for h in hs:
        text = open(h).read()
        if f"){delim}\"" in text:
            raise RuntimeError(f"{h} contains the raw-string delimiter")
        parts.append(f'R"{delim}({text}){delim}"')
    names = ", ".join(f'"{h}"' for h in JIT_HEADERS)
    with open(src, "w") as f:
        f.write("// generated by build.py: device headers for run-time compiled kernels\n")
        f.write("namespace prism {\n")
        f.write(f"extern const int kJitHeaderCount = {len(hs)};\n")
        f.write(f"extern const char* const kJitHeaderNames[] = {{{names}}};\n")
        f.write("extern const char* const kJitHeaderTexts[] = {\n" + ",\n".join(parts) + "};\n}\n")
    r = subprocess.run(["g++", "-O1", "-fPIC", "-c", src, "-o", obj], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"embedding device headers failed:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, debug: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-DPRISM_DEBUG=1"] if debug else []
    if verbose:
        extra += ["-Xptxas", "-v"]
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force, extra), sources()))
    objs.append(jit_headers_object(force))
    if force or not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", *objs, "-o", OUT, "-lpthread", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, debug="--debug" in sys.argv, verbose="-v" in sys.argv))
