"""Build the native library and CLI in-tree (sm_100a).

Outputs (git-ignored, shipped with the tree):
  gahhg_b200/libgahhg.so   C ABI declared in include/gahhg.h
  gahhg_b200/gahhg         command-line drop-in for GPISP.exe

Every CUDA source is compiled with ``--fmad=false`` and host C++ with
``-ffp-contract=off``: only explicit fma() calls fuse, so the FP64 arithmetic
of the reference-semantics path and the canonical conversion give the same
bits on the CPU and the GPU.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgahhg.so")
CLI = os.path.join(HERE, "gahhg")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_FLAGS = ARCH + ["-O3", "-std=c++17", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC",
                   "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr",
                   "-I", os.path.join(REPO, "include"), "-I", CSRC]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
             "-I", os.path.join(REPO, "include"), "-I", CSRC, "-I", "/usr/local/cuda/include"]


def _sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp") and f != "cli.cpp")
    return cu, cpp


def _stale(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    inc = os.path.join(REPO, "include")
    hs += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    return hs


def _compile(args):
    cmd, out = args
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return out


def build(verbose=False, jobs=None):
    os.makedirs(OBJ, exist_ok=True)
    cu, cpp = _sources()
    hdrs = _headers()
    jobsl = []
    objs = []
    for f in cu:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f + ".o")
        objs.append(obj)
        if _stale(obj, [src] + hdrs):
            jobsl.append(([NVCC] + CU_FLAGS + ["-c", src, "-o", obj], obj))
    for f in cpp + ["cli.cpp"]:
        src = os.path.join(CSRC, f)
        obj = os.path.join(OBJ, f + ".o")
        if f != "cli.cpp":
            objs.append(obj)
        if _stale(obj, [src] + hdrs):
            jobsl.append((["g++"] + CXX_FLAGS + ["-c", src, "-o", obj], obj))
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count()) as ex:
        for out in ex.map(_compile, jobsl):
            if verbose:
                print("built", os.path.relpath(out, REPO))
    if _stale(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB + ".tmp"] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        _compile((cmd, LIB))
        os.replace(LIB + ".tmp", LIB)
    cli_obj = os.path.join(OBJ, "cli.cpp.o")
    if _stale(CLI, [cli_obj, LIB]):
        cmd = ["g++", "-o", CLI + ".tmp", cli_obj, "-L", HERE, "-lgahhg", "-Wl,-rpath,$ORIGIN"]
        _compile((cmd, CLI))
        os.replace(CLI + ".tmp", CLI)
    return LIB, CLI


if __name__ == "__main__":
    print(build(verbose=True))
