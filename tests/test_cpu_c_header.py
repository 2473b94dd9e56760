"""include/gahhg.h as a C caller sees it: a strict C99 program (as a cgo or
other C FFI binding would compile) includes the header with -pedantic and
-Werror, links the in-tree libgahhg.so and calls the entry points that need
no GPU: ABI version, knobs, build options, the POLYGON loader and its error
path.  Host only."""
import os
import shutil
import subprocess

import pytest

from tests.conftest import REPO

PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "gahhg.h"

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    if (gahhg_abi_version() < 1) return 3;
    if (gahhg_get_knob(GAHHG_KNOB_GROUPED_PASS2) != 0) return 4;
    if (gahhg_set_knob(GAHHG_KNOB_GROUPED_PASS2, 3) != GAHHG_OK) return 5;
    if (gahhg_get_knob(GAHHG_KNOB_GROUPED_PASS2) != 3) return 6;
    if (gahhg_set_knob(GAHHG_KNOB_GROUPED_PASS2, 4) == GAHHG_OK) return 7;
    if (strlen(gahhg_last_error()) == 0) return 8;
    gahhg_set_knob(GAHHG_KNOB_GROUPED_PASS2, 0);
    gahhg_build_opts o;
    gahhg_build_opts_init(&o);
    if (o.semantics != GAHHG_SEMANTICS_EXACT) return 9;
    gahhg_polygon* p = NULL;
    if (gahhg_polygon_load(argv[1], &p) != GAHHG_OK || !p) return 10;
    printf("edges %d\n", gahhg_polygon_num_edges(p));
    gahhg_polygon_free(p);
    gahhg_polygon* q = NULL;
    if (gahhg_polygon_load(argv[2], &q) == GAHHG_OK) return 11;
    printf("error %s\n", gahhg_last_error());
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_header_is_c99_and_library_links(tmp_path):
    lib = os.path.join(REPO, "gahhg_b200", "libgahhg.so")
    if not os.path.exists(lib):
        pytest.skip("libgahhg.so not built")
    src = tmp_path / "caller.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "caller"
    libdir = os.path.dirname(lib)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I",
                    os.path.join(REPO, "include"), str(src), "-o", str(exe), "-L", libdir, "-lgahhg",
                    "-Wl,-rpath," + libdir], check=True, capture_output=True, text=True)
    good = tmp_path / "square.txt"
    good.write_text("POLYGON 1 0\n0 5\n0 0\n1 0\n1 1\n0 1\n0 0\n")
    bad = tmp_path / "bad.txt"
    bad.write_text("POLYGON 1 0\n0 5\n0 0\n1 0\n")
    r = subprocess.run([str(exe), str(good), str(bad)], capture_output=True, text=True, timeout=60,
                       env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    assert "edges 4" in r.stdout
    assert "error " in r.stdout
