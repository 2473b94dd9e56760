"""Recipe: build the reference's own GAHHG code for the CPU (test oracle).

TEST INFRASTRUCTURE.  Reads the reference sources where they lie
(``/root/reference/source``), never copies them into the repository, and writes
only build outputs into ``oracle/_ref/`` (git-ignored):

  oracle/_ref/libgahhg_ref.so   reference kernels + host code + ref_harness.cpp
  oracle/_ref/gpisp_ref         the reference command-line program (GPISP.cu)

The sources are CUDA C++; three mechanical edits, made in a temporary
directory that is deleted afterwards, let g++ build them:

  1. launch syntax ``kernel << <b, t >> > (args)`` -> ``REFSHIM_LAUNCH(kernel,
     b, t)(args)`` (refshim.h runs every thread index on the CPU);
  2. source/GPISPPolygon.cu:200 ``for (int j = 0; j < inVNum[i]; i++)``
     increments ``i`` instead of ``j`` and reads past the ring arrays when the
     polygon has holes (undefined behaviour, result unused) -> ``j++``;
  3. nothing else: Windows and CUDA headers are replaced by the stand-ins in
     ``oracle/refshim`` via the include path.

The level-0 grid, whose only implementation is a closed library, comes from
``oracle/refshim/ref_grid0.cpp``; the missing scan utilities from refshim.cpp.
Compiled with ``-O2 -ffp-contract=off`` so no multiply-add is fused.
"""
import os
import re
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
SHIM = os.path.join(HERE, "refshim")
# The reference checkout: $GAHHG_REFERENCE (default /root/reference); its
# sources are under source/.
REFERENCE_ROOT = os.environ.get("GAHHG_REFERENCE", "/root/reference")
DEFAULT_SRC = os.path.join(REFERENCE_ROOT, "source")

LAUNCH_RE = re.compile(r"(\w+)\s*<<\s*<\s*(.+?)\s*>>\s*>\s*\(")
BBOX_BUG = "for (int j = 0; j < inVNum[i]; i++)"
BBOX_FIX = "for (int j = 0; j < inVNum[i]; j++)"

SOURCES = ["GPISPAHHG.cu", "GPISPPolygon.cu", "GPISPTP.cu", "GPISP.cu"]
HEADERS = ["GPISPAHHG.cuh", "GPISPDS.cuh", "GPISPParam.h", "GPISPPolygon.cuh",
           "GPISPTP.cuh", "common.h"]


def _transform(text, name):
    text = LAUNCH_RE.sub(lambda m: "REFSHIM_LAUNCH(%s, %s)(" % (m.group(1), m.group(2)), text)
    if name == "GPISPPolygon.cu":
        if BBOX_BUG not in text:
            raise RuntimeError("GPISPPolygon.cu: expected loop not found")
        text = text.replace(BBOX_BUG, BBOX_FIX)
    if "<<<" in text or "<< <" in text:
        raise RuntimeError("%s: launch left untranslated" % name)
    return text


def _read(path):
    with open(path, "rb") as f:
        data = f.read()
    if data.startswith(b"\xef\xbb\xbf"):
        data = data[3:]
    return data.decode("utf-8", errors="replace")


def build(src=DEFAULT_SRC, out=OUT, verbose=False):
    if not os.path.isdir(src):
        raise FileNotFoundError("reference sources not found at %s" % src)
    os.makedirs(out, exist_ok=True)
    tmp = tempfile.mkdtemp(prefix="gahhg_ref_")
    try:
        os.makedirs(os.path.join(tmp, "scan"))
        for h in HEADERS:
            with open(os.path.join(tmp, h), "w") as f:
                f.write(_read(os.path.join(src, h)))
        with open(os.path.join(tmp, "scan", "scan.cuh"), "w") as f:
            f.write("#pragma once\nvoid myscan(int* output, int* input, int length, bool bcao);\n")
        for s in SOURCES:
            with open(os.path.join(tmp, s), "w") as f:
                f.write(_transform(_read(os.path.join(src, s)), s))
        flags = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-w",
                 "-I", tmp, "-I", SHIM, "-I", os.path.join(REPO, "include"),
                 "-include", os.path.join(SHIM, "refshim.h")]
        common = [os.path.join(SHIM, "refshim.cpp"), os.path.join(SHIM, "ref_grid0.cpp")]
        ref_cu = [os.path.join(tmp, s) for s in SOURCES if s != "GPISP.cu"]
        lib = os.path.join(out, "libgahhg_ref.so")
        cmd = flags + ["-shared", "-o", lib + ".tmp"] + common + \
            ["-x", "c++"] + ref_cu + [os.path.join(SHIM, "ref_harness.cpp")]
        # ref_harness.cpp must not be read as CUDA; -x c++ applies to all anyway
        subprocess.run(cmd, check=True, capture_output=not verbose)
        os.replace(lib + ".tmp", lib)
        exe = os.path.join(out, "gpisp_ref")
        cmd = flags + ["-o", exe + ".tmp"] + common + ["-x", "c++"] + \
            [os.path.join(tmp, s) for s in SOURCES]
        subprocess.run(cmd, check=True, capture_output=not verbose)
        os.replace(exe + ".tmp", exe)
        return lib, exe
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else DEFAULT_SRC
    print(build(src, verbose=True))
