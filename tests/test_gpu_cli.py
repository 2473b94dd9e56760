"""The `gahhg` command line against the reference program built for the CPU
(oracle/_ref/gpisp_ref): same flags, same result CSV byte for byte, same
report block except the date and the timings."""
import os
import re
import subprocess

import numpy as np
import pytest

from tests.golden.fixtures import key

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(REPO, "gahhg_b200", "gahhg")

CASES = [("various/Square_72.txt", "Square_72_query.csv"), ("various/Radiometer.txt", "Radiometer_query.csv"),
         ("various/Tennessee.txt", "Tennessee_query.csv"), ("various/NA0.txt", "uniform"),
         ("Mars/100.txt", "Mars_query.csv")]


def _strip(report):
    out = []
    for ln in report.splitlines():
        if ln.startswith("-----") or ln.startswith("Time of") or ln.startswith("Total test time") \
                or ln.startswith("Average test time"):
            continue
        out.append(re.sub(r"/tmp/\S+/", "", ln))
    return out


@pytest.mark.parametrize("poly,query", CASES)
def test_cli_matches_reference_program(oracle_ref, inputs, tmp_path, poly, query):
    pfile = inputs.polygon_file(poly, tmp_path)
    qfile = inputs.query_file(query, tmp_path)
    outs = {}
    for tag, exe in (("ours", CLI), ("ref", oracle_ref.REF_EXE)):
        rep = tmp_path / ("%s_report.txt" % tag)
        res = tmp_path / ("%s_result.csv" % tag)
        p = subprocess.run([exe, "/polyfile", pfile, "/tpfile", qfile, "/reportfile", str(rep),
                            "/resultfile", str(res)], capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stderr
        outs[tag] = (p.stdout, rep.read_text(), res.read_bytes())
    assert outs["ours"][2] == outs["ref"][2]
    assert _strip(outs["ours"][1]) == _strip(outs["ref"][1])
    # same progress messages
    assert outs["ours"][0].splitlines()[:2] == outs["ref"][0].splitlines()[:2]


def test_cli_loader_failure_exit_code(tmp_path):
    bad = tmp_path / "bad.txt"
    bad.write_text("POLYGON 2 0\n")
    p = subprocess.run([CLI, "/polyfile", str(bad), "/tpfile", "x.csv"], capture_output=True, text=True)
    assert p.returncode == 255  # main returns -1
    assert "Error. Line 1 of %s. Wrong format." % bad in p.stdout
