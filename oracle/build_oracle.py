"""Build the exact oracle (oracle/exact_pip.c) -> oracle/_build/liboracle_exact.so.

TEST INFRASTRUCTURE.  Plain C, gcc, no fused multiply-add except the explicit
fma() of the error-free products.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_build", "liboracle_exact.so")


def build():
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
