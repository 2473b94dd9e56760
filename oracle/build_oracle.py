"""Build the exact oracle (oracle/exact_pip.c) -> oracle/_build/liboracle_exact.so,
and its GPU brute force (oracle/brute_gpu.cu) -> oracle/_build/liboracle_brute.so.

TEST INFRASTRUCTURE.  Plain C, gcc, no fused multiply-add except the explicit
fma() of the error-free products; the GPU brute force likewise (nvcc
--fmad=false), for sm_100a.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_build", "liboracle_exact.so")
BRUTE = os.path.join(HERE, "_build", "liboracle_brute.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def _fresh(out, deps):
    return os.path.exists(out) and os.path.getmtime(out) > max(os.path.getmtime(d) for d in deps)


def build_brute():
    src = os.path.join(HERE, "brute_gpu.cu")
    canon = os.path.join(REPO, "include", "gahhg_canon.h")
    if _fresh(BRUTE, [src, canon]):
        return BRUTE
    os.makedirs(os.path.dirname(BRUTE), exist_ok=True)
    subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "--fmad=false",
                    "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-shared",
                    "-I", os.path.join(REPO, "include"), src, "-o", BRUTE + ".tmp", "-lcudart_static", "-lrt",
                    "-ldl", "-lpthread"], check=True)
    os.replace(BRUTE + ".tmp", BRUTE)
    return BRUTE


def build():
    build_brute()
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    src = os.path.join(HERE, "exact_pip.c")
    if os.path.exists(OUT) and os.path.getmtime(OUT) > max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(REPO, "include", "gahhg_canon.h"))):
        return OUT
    subprocess.run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
                    "-Wall", "-I", os.path.join(REPO, "include"), src, "-o", OUT + ".tmp", "-lm"], check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build())
