"""The CSV point loader (GPISPTP::loadTPFromCSV, source/GPISPTP.cu:13-79):
parsed by all host threads, it must give the values and the rejected line of
the reference's serial sscanf("%lf,%lf") reading (the platform's C library,
as in the reference built for the CPU here), on small files (one thread) and on
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
        ("1e,2", (1.0, 2.0)),                          # glibc's %lf, as the reference built here: "1e" -> 1
        ("1.5e-,3", (1.5, 3.0)),
        ("0x,1", None),                                # no digits after "0x": rejected
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


# ---- POLYGON files large enough for the threaded vertex parse ------------

def _big_polygon_lines():
    """A 200,000-vertex outer ring and three holes as POLYGON text lines,
    with some vertex lines in the forms that only the serial "%lf %lf"
    reading handles (a '+' sign, hex, tabs, CRLF, trailing text, no space
    before a minus sign)."""
    from gahhg_b200 import synth
    rng = np.random.default_rng(31)
    rings = [synth.star_ring(40.0, -10.0, 200_000, 20.0, 0.2, rng)]
    for k in range(3):
        rings.append(synth.star_ring(40.0 + 4.0 * (k - 1), -10.0, 5_000 + k, 1.0, 0.1, rng)[::-1])
    lines = ["POLYGON 1 %d" % (len(rings) - 1)]
    for i, r in enumerate(rings):
        lines.append("%d %d" % (i, len(r) + 1))
        lines += ["%.17g %.17g" % (lo, la) for lo, la in np.concatenate([r, r[:1]])]
    for at, form in [(10, "+{} {}"), (50_001, "{}\t{}"), (120_000, "{} {}\r"), (150_000, "{}  {} trailing"),
                     (180_000, "  {} {}")]:
        lo, la = (float(x) for x in lines[at].split())
        lines[at] = form.format(repr(lo), repr(la))
    lines[70_000] = "%s %s" % (float(lines[70_000].split()[0]).hex(), lines[70_000].split()[1])
    lo, la = (float(x) for x in lines[90_000].split())
    lines[90_000] = "%r%r" % (lo, -abs(la)) if la != 0 else lines[90_000]
    return lines


@pytest.fixture(scope="module")
def big_polygon_lines():
    return _big_polygon_lines()


def _write_lines(path, lines, final_newline=True):
    with open(path, "w", newline="") as f:
        f.write("\n".join(lines) + ("\n" if final_newline else ""))


def test_large_polygon_matches_reference(big_polygon_lines, tmp_path, oracle_ref):
    path = str(tmp_path / "big.txt")
    _write_lines(path, big_polygon_lines)
    P = G.Polygon.from_file(path)
    xyz, pe = P.export()
    assert len(xyz) == 200_000 + 5_000 + 5_001 + 5_002
    rx, rp = oracle_ref.RefGPISP(path, maxdepth=1).polygon()
    assert np.array_equal(xyz, rx) and np.array_equal(pe, rp)
    # no final newline: same polygon
    _write_lines(path, big_polygon_lines, final_newline=False)
    x2, p2 = G.Polygon.from_file(path).export()
    assert np.array_equal(x2, rx) and np.array_equal(p2, rp)


def test_large_polygon_first_error(big_polygon_lines, tmp_path, capfd, oracle_ref):
    """Wherever the faults are, the message names the first one in file order,
    as the reference's serial reading does."""
    hole1 = 2 + 200_001          # 0-based line of the first hole's header
    cases = [
        {150_000: "1.0 x"},                            # a vertex line of the outer ring
        {hole1 + 3: "nan?", 199_000: "1,2"},            # two faults: the earlier one counts
        {hole1: "1 3"},                                 # a hole with too few vertices
        {hole1 + 5_002: "junk"},                        # the second hole's header
        {hole1 + 5_002: "junk", 60_000: "1e 2"},        # a vertex fault before a header fault
        {"truncate": hole1 + 5_002 + 100},              # the file ends inside a hole
    ]
    for case in cases:
        lines = list(big_polygon_lines)
        if "truncate" in case:
            lines = lines[:case["truncate"]]
        else:
            for at, text in case.items():
                lines[at] = text
        path = str(tmp_path / "bad.txt")
        _write_lines(path, lines)
        with pytest.raises(G.GahhgError):
            G.Polygon.from_file(path)
        ours = [l for l in capfd.readouterr().out.splitlines() if l.startswith("Error.")]
        with pytest.raises(ValueError):
            oracle_ref.RefGPISP(path, maxdepth=1)
        ref = [l for l in capfd.readouterr().out.splitlines() if l.startswith("Error.")]
        assert ours == ref and len(ours) == 1, (case, ours, ref)


@pytest.mark.parametrize("text", [
    "",                                                     # empty file
    "POLYGON 1 0\n",                                        # header only
    "POLYGON 1 0",                                          # one line, no newline: getline keeps size - 1 chars
    "POLYGON 1 12",                                         # the same, with a count the cut shortens
    "POLYGON 1 1\n0 5\n0 0\n10 0\n10 10\n0 10\n0 0",        # a hole announced, the file ends
    "POLYGON 1 0\r\n0 5\r\n0 0\r\n10 0\r\n10 10\r\n0 10\r\n0 0\r\n",   # CRLF lines
    "POLYGON 1 0\n0 5 extra\n0 0\n10 0\n10 10\n0 10\n0 0",  # text after the count, no final newline
    "POLYGON 1 0\n0 5\n0 0\n10 0\n10 10\n0 10\n",           # one vertex line short
])
def test_polygon_edge_cases_match_reference(text, tmp_path, capfd, oracle_ref):
    path = str(tmp_path / "p.txt")
    with open(path, "w", newline="") as f:
        f.write(text)
    try:
        ours = G.Polygon.from_file(path).export()
    except G.GahhgError:
        ours = None
    out_ours = [l for l in capfd.readouterr().out.splitlines() if l.startswith("Error.")]
    try:
        ref = oracle_ref.RefGPISP(path, maxdepth=1).polygon()
    except ValueError:
        ref = None
    out_ref = [l for l in capfd.readouterr().out.splitlines() if l.startswith("Error.")]
    assert out_ours == out_ref
    assert (ours is None) == (ref is None)
    if ours is not None:
        assert np.array_equal(ours[0], ref[0]) and np.array_equal(ours[1], ref[1])


@pytest.mark.parametrize("text", ["1,2", "1,2\n", "1,2\n3,4", "1,2\r3,4\r", "170.5,-3.25 tail", "x,y"])
def test_points_line_ends_match_reference_program(text, tmp_path, oracle_ref):
    """The number of points the reference program reads (its result CSV has
    one line per point) for files whose last line has no line end: a file
    without any '\\n' is read as no points, since getline(buf, size) stores
    at most size - 1 characters of its only line and then fails."""
    import subprocess
    poly = tmp_path / "sq.txt"
    poly.write_text("POLYGON 1 0\n0 5\n0 0\n10 0\n10 10\n0 10\n0 0\n")
    csv = tmp_path / "q.csv"
    with open(csv, "w", newline="") as f:
        f.write(text)
    res = tmp_path / "res.csv"
    r = subprocess.run([oracle_ref.REF_EXE, "/polyfile", str(poly), "/tpfile", str(csv), "/reportfile",
                        str(tmp_path / "rep.txt"), "/resultfile", str(res)], capture_output=True, text=True,
                       timeout=120, cwd=str(tmp_path))
    try:
        ours = len(G.load_points(str(csv)))
    except G.GahhgError:
        ours = None
    if r.returncode != 0:
        assert ours is None, (text, r.stdout)
        return
    with open(res) as f:
        assert ours == len(f.read().splitlines()), (text, ours)


def test_points_files_match_reference_program(tmp_path, oracle_ref):
    """Seeded files of valid and malformed lines (other separators, blanks,
    signs, hex, exponents, trailing text, CR LF ends, a missing last line
    end): the reference program built for the CPU and this loader accept the
    same files with the same number of points, or name the same first bad
    line."""
    import random
    import re
    import subprocess
    forms = ["1.5,2.5", "-10.25,3e-3", "\t-1,2", "+4,5", "0x1p3,7", "1e,2", "1;2", "1 2", "", " ", "a,b",
             "12,13,14", "5,6 junk", "inf,-inf", "3,", ",3", "170.123456789012345,-0.5", "-0,0", "1e308,1e-308"]
    poly = tmp_path / "sq.txt"
    poly.write_text("POLYGON 1 0\n0 5\n0 0\n10 0\n10 10\n0 10\n0 0\n")
    rng = random.Random(4242)
    csv = tmp_path / "q.csv"
    res = tmp_path / "res.csv"
    for case in range(150):
        lines = [rng.choice(forms) for _ in range(rng.randint(1, 6))]
        sep = rng.choice(["\n", "\n", "\r\n"])
        text = sep.join(lines) + (sep if rng.random() < 0.7 else "")
        with open(csv, "w", newline="") as f:
            f.write(text)
        if res.exists():
            res.unlink()
        r = subprocess.run([oracle_ref.REF_EXE, "/polyfile", str(poly), "/tpfile", str(csv), "/reportfile",
                            str(tmp_path / "rep.txt"), "/resultfile", str(res)], capture_output=True, text=True,
                           timeout=120, cwd=str(tmp_path))
        m = re.search(r"Error\. Line (\d+) of .*\. Wrong format\.", r.stdout)
        try:
            ours = len(G.load_points(str(csv)))
            ours_bad = None
        except G.GahhgError as e:
            ours = None
            ours_bad = int(re.search(r"line (\d+) ", str(e)).group(1))
        if m:
            assert ours_bad == int(m.group(1)), (case, repr(text), ours_bad, m.group(1))
        else:
            assert r.returncode == 0 and ours is not None, (case, repr(text), r.stdout[-300:])
            with open(res) as f:
                assert ours == len(f.read().splitlines()), (case, repr(text), ours)
