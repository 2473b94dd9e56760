"""The POLYGON loader (GPISPPolygon::loadPolyFromTXT,
source/GPISPPolygon.cu:32-278) against the reference's own loader built for
the CPU, on seeded mutations of a small two-ring file: deleted, repeated,
truncated and blank lines, changed counts, junk tokens, other separators,
leading and trailing white space, CR LF line ends, a missing final newline.
For each file both loaders must accept it with the same vertices and edges,
or both reject it with the same "Error. Line ..." message.

Negative counts are left out: the reference allocates arrays of that size
and aborts (std::bad_array_new_length on a negative hole count); this
loader rejects such a file with an error message of the reference's form
(test_negative_counts_are_rejected).  Host only.
"""
import random

import numpy as np
import pytest

import gahhg_b200 as G

BASE = ["POLYGON 1 1", "0 9", "0 0", "10 0", "20 5", "20 15", "10 20", "0 20", "-5 10", "0 0",
        "1 6", "5 5", "5 10", "10 10", "10 5", "5 5"]
JUNK = ["x", "1", "1 2 3", "", " ", "nan nan", "1e400 2", "0x10 3", "+1 -2", "1\t2", "-1-2", "POLYGON 1 0",
        "0 3", "0 2", "2 5"]
HEADERS = ["POLYGON 1 0", "POLYGON 1 2", "POLYGON 2 1", "POLYGON 0 1", "polygon 1 1", "POLYGON 1",
           "POLYGON 1 1 1", "POLYGON1 1"]


def mutate(rng):
    lines = list(BASE)
    for _ in range(rng.randint(1, 3)):
        if not lines:
            break
        k = rng.randrange(len(lines))
        op = rng.randrange(12)
        if op == 0:
            del lines[k]
        elif op == 1:
            lines.insert(k, lines[k])
        elif op == 2:
            lines[k] = rng.choice(JUNK)
        elif op == 3:
            t = lines[k].split()
            if t:
                t[rng.randrange(len(t))] = str(rng.choice([0, 1, 2, 3, 4, 5, 8, 9, 10, 100]))
            lines[k] = " ".join(t)
        elif op == 4:
            lines.insert(k, "")
        elif op == 5:
            lines = lines[:k]
        elif op == 6:
            lines[k] = lines[k] + rng.choice([" trailing", "\t", " 7", ",", "\r"])
        elif op == 7:
            lines[k] = rng.choice(["  ", "\t"]) + lines[k]
        elif op == 8:
            lines[k] = lines[k].replace(" ", rng.choice(["  ", "\t", ",", ";"]))
        elif op == 9:
            lines[0] = rng.choice(HEADERS)
        elif op == 10:
            lines[k] = lines[k][: rng.randrange(len(lines[k]) + 1)]
        else:
            lines.append(rng.choice(["", "junk", "1 1"]))
    sep = rng.choice(["\n", "\n", "\r\n"])
    return sep.join(lines) + (sep if rng.random() < 0.8 else "")


def _load(fn, capfd, exc):
    try:
        res = fn()
    except exc:
        res = None
    msgs = [l for l in capfd.readouterr().out.splitlines() if l.startswith("Error.")]
    return res, msgs


def test_mutated_polygon_files_match_reference(tmp_path, capfd, oracle_ref):
    rng = random.Random(20261204)
    path = str(tmp_path / "m.txt")
    accepted = rejected = 0
    for case in range(400):
        text = mutate(rng)
        with open(path, "w", newline="") as f:
            f.write(text)
        ours, ours_msg = _load(lambda: G.Polygon.from_file(path).export(), capfd, G.GahhgError)
        ref, ref_msg = _load(lambda: oracle_ref.RefGPISP(path, maxdepth=1).polygon(), capfd, ValueError)
        assert ours_msg == ref_msg, (case, text, ours_msg, ref_msg)
        assert (ours is None) == (ref is None), (case, text)
        if ours is None:
            rejected += 1
            continue
        accepted += 1
        assert np.array_equal(ours[0], ref[0]) and np.array_equal(ours[1], ref[1]), (case, text)
    assert accepted > 20 and rejected > 100  # both outcomes are exercised


@pytest.mark.parametrize("text", ["POLYGON 1 -1\n" + "\n".join(BASE[1:10]) + "\n",
                                  "POLYGON 1 0\n0 -3\n0 0\n1 0\n1 1\n"])
def test_negative_counts_are_rejected(text, tmp_path, capfd):
    path = str(tmp_path / "n.txt")
    with open(path, "w") as f:
        f.write(text)
    with pytest.raises(G.GahhgError):
        G.Polygon.from_file(path)
    assert any(l.startswith("Error. Line ") for l in capfd.readouterr().out.splitlines())
