"""The CSV point loader (GPISPTP::loadTPFromCSV, source/GPISPTP.cu:13-79):
parsed by all host threads, it must give the values and the rejected line of
the reference's serial "%lf,%lf" reading, on small files (one thread) and on
files large enough to be split into chunks; binary sidecars must round-trip
and be ignored once the CSV changes.  Host code only.
"""
import math
import os

import numpy as np
import pytest

import gahhg_b200 as G
from gahhg_b200 import _lib


def _write(path, text):
    with open(path, "w", newline="") as f:
        f.write(text)


def test_line_forms(tmp_path):
    lines = [
        ("1.5,2.5", (1.5, 2.5)),
        (" -10.25 ,\t3e-3", None),                    # space before ',' : rejected by "%lf,%lf"
        ("\t-10.25,\t3e-3", (-10.25, 3e-3)),           # leading white space is skipped
        ("+4,5", (4.0, 5.0)),                          # '+' sign
        ("0x1p3,7", (8.0, 7.0)),                       # hexadecimal floating point
        ("7,0x1p-2", (7.0, 0.25)),
        ("180.000001,-90.000000\r", (180.000001, -90.0)),  # CRLF files
        ("12,13,14", (12.0, 13.0)),                    # anything after the second number is ignored
        ("5,6 junk", (5.0, 6.0)),
        ("1e,2", None),                                # "1" then 'e': not followed by ','
        ("0.1,1e-320", (0.1, 1e-320)),                 # subnormal
        ("inf,-inf", (math.inf, -math.inf)),
        ("170.12345678901234567,-0.000000000000000001", (170.12345678901234567, -1e-18)),
    ]
    for k, (text, want) in enumerate(lines):
        path = str(tmp_path / ("l%d.csv" % k))
        _write(path, text + "\n")
        if want is None:
            with pytest.raises(G.GahhgError):
                G.load_points(path)
            continue
        got = G.load_points(path)
        assert got.shape == (1, 2), text
        assert got[0, 0] == want[0] and got[0, 1] == want[1], (text, got)


def test_rejected_lines(tmp_path):
    for text, bad in [("1,2\n\n3,4\n", 2), ("1,2\n3,\n", 2), ("a,b\n", 1), ("1;2\n", 1), ("1 2\n", 1),
                      ("1,2\n3,4", None), ("", None), ("1,2\n,3\n", 2)]:
        path = str(tmp_path / "r.csv")
        _write(path, text)
        if bad is None:
            n = len(G.load_points(path))
            assert n == text.count("\n") + (1 if text and not text.endswith("\n") else 0)
            continue
        with pytest.raises(G.GahhgError) as e:
            G.load_points(path)
        assert ("line %d " % bad) in str(e.value), (text, str(e.value))


def test_large_file_in_chunks(tmp_path):
    rng = np.random.default_rng(7)
    n = 700_000  # ~26 MB: several chunks
    ll = np.stack([rng.uniform(-180, 180, n), rng.uniform(-90, 90, n)], 1)
    text = "".join("%.17g,%.17g\n" % (a, b) for a, b in ll)
    path = str(tmp_path / "big.csv")
    _write(path, text)
    assert os.path.getsize(path) > 3 * (4 << 20)
    got = G.load_points(path)
    assert np.array_equal(got, ll)
    # the first of two bad lines, wherever the chunks fall
    rows = text.splitlines(keepends=True)
    for first, second in [(123_457, 600_001), (500_000, 500_001), (1, 699_999)]:
        bad_rows = list(rows)
        bad_rows[first - 1] = "x,1\n"
        bad_rows[second - 1] = "1;2\n"
        _write(path, "".join(bad_rows))
        with pytest.raises(G.GahhgError) as e:
            G.load_points(path)
        assert ("line %d " % first) in str(e.value)


def test_sidecar(tmp_path):
    rng = np.random.default_rng(8)
    ll = np.round(np.stack([rng.uniform(-180, 180, 5000), rng.uniform(-90, 90, 5000)], 1), 6)
    path = str(tmp_path / "q.csv")
    _write(path, "".join("%.6f,%.6f\n" % (a, b) for a, b in ll))
    first = G.load_points(path, sidecar=True)      # parses and writes q.csv.f64
    assert os.path.exists(path + ".f64")
    assert os.path.getsize(path + ".f64") == 64 + 16 * len(ll)
    again = G.load_points(path, sidecar=True)      # reads the sidecar
    assert np.array_equal(first, again) and np.array_equal(first, G.load_points(path))
    # a changed CSV makes the sidecar stale: the CSV is parsed again
    _write(path, "1,2\n")
    assert np.array_equal(G.load_points(path, sidecar=True), [[1.0, 2.0]])
    assert os.path.getsize(path + ".f64") == 64 + 16
    # a sidecar alone is never used without its CSV
    os.unlink(path)
    with pytest.raises(G.GahhgError) as e:
        G.load_points(path, sidecar=True)
    assert e.value.status == _lib.ERR_IO
