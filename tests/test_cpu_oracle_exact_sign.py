"""The exact oracle's orientation predicate (oracle/exact_pip.c:
orient_raw = FP64 filter + Shewchuk expansion, then simulation of
simplicity) against exact rational arithmetic: sign(a . (b x c)) computed
with fractions.Fraction from the same doubles.  Random, near-coplanar
(perturbed down to 1e-18), great-circle midpoint and exactly coplanar
triples.  With simulation of simplicity the sign must equal the exact sign
wherever that is not zero, never be zero for three distinct points (two
identical points give 0: the callers apply the vertex rule before), and flip
when two arguments are exchanged.  The kernels' own predicate header
(gahhg_b200/csrc/exact_pred.cuh, built for the host) is held to the same
rational signs and to the oracle's separately written simulation of
simplicity.  Host only; pins the oracle that every exact-label test relies
on, and the exact tier's arithmetic.
"""
import ctypes
import os
import subprocess
from fractions import Fraction

import numpy as np
import pytest

from oracle import exact

HERE = os.path.dirname(os.path.abspath(__file__))


def _exact_sign(a, b, c):
    a, b, c = ([Fraction(float(x)) for x in v] for v in (a, b, c))
    d = (a[0] * (b[1] * c[2] - b[2] * c[1]) + a[1] * (b[2] * c[0] - b[0] * c[2]) +
         a[2] * (b[0] * c[1] - b[1] * c[0]))
    return (d > 0) - (d < 0)


def _unit(v):
    return v / np.linalg.norm(v)


def _triples(n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        kind = i % 5
        a, b = _unit(rng.normal(size=3)), _unit(rng.normal(size=3))
        if kind == 0:
            c = _unit(rng.normal(size=3))
        elif kind == 1:   # near the plane of a and b, offsets 1e-18 .. 1e-8
            c = _unit(a * rng.uniform(-1, 1) + b * rng.uniform(-1, 1)) + rng.normal(size=3) * 10.0 ** rng.uniform(-18, -8)
        elif kind == 2:   # the midpoint of the arc, rounded: det is a few ulps or zero
            c = _unit(a + b)
        elif kind == 3:   # exactly coplanar small integers, scaled by a power of two
            m = rng.integers(-50, 50, size=(2, 3)).astype(np.float64)
            s = 2.0 ** int(rng.integers(-20, 20))
            a, b = m[0] * s, m[1] * s
            c = (m[0] * int(rng.integers(-5, 5)) + m[1] * int(rng.integers(-5, 5))) * s
        else:             # nearly parallel a and b (short edges), c near them
            b = _unit(a + rng.normal(size=3) * 10.0 ** rng.uniform(-12, -6))
            c = _unit(a + (b - a) * rng.uniform(-2, 3) + rng.normal(size=3) * 10.0 ** rng.uniform(-20, -12))
        out.append((np.asarray(a, np.float64), np.asarray(b, np.float64), np.asarray(c, np.float64)))
    return out


def test_orient_matches_rational_arithmetic():
    zeros = nonzero_near = 0
    for i, (a, b, c) in enumerate(_triples(15_000, 97)):
        want = _exact_sign(a, b, c)
        got = exact.orient(a, b, c, sos=False)
        assert got == want, (i, a.tolist(), b.tolist(), c.tolist(), got, want)
        s = exact.orient(a, b, c, sos=True)
        if want != 0:
            assert s == want, i
            if i % 5 in (1, 2, 4):
                nonzero_near += 1
        elif (a == b).all() or (b == c).all() or (a == c).all():
            assert s == 0, i  # identical points: no perturbation orders them (callers test them first)
        else:
            zeros += 1
            assert s in (-1, 1), i
            assert exact.orient(b, a, c, sos=True) == -s, i
            assert exact.orient(a, c, b, sos=True) == -s, i
            assert exact.orient(b, c, a, sos=True) == s, i
    # both the exact-zero and the near-degenerate branches were exercised
    assert zeros > 1000 and nonzero_near > 5000


@pytest.fixture(scope="module")
def kernel_signs(tmp_path_factory):
    """The kernels' predicate header (gahhg_b200/csrc/exact_pred.cuh) built
    for the host: (exact sign by expansions, orient with simulation of
    simplicity) per triple."""
    out = str(tmp_path_factory.mktemp("pred") / "libpred_probe.so")
    subprocess.check_call(["g++", "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-I",
                           os.path.join(os.path.dirname(HERE), "include"), "-o", out,
                           os.path.join(HERE, "native", "pred_probe.cpp")])
    lib = ctypes.CDLL(out)
    lib.exact_signs.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p]
    lib.exact_signs.restype = None

    def signs(triples):
        xyz = np.ascontiguousarray(np.array([np.concatenate(t) for t in triples]), dtype=np.float64)
        res = np.zeros((len(triples), 2), dtype=np.int32)
        lib.exact_signs(xyz.ctypes.data, len(triples), res.ctypes.data)
        return res
    return signs


def test_kernel_predicate_matches_rational_arithmetic_and_oracle(kernel_signs):
    """The exact tier's own code (the header the kernels compile), built for
    the host: its expansion sign equals rational arithmetic, and its
    simulation of simplicity equals the oracle's separately written one."""
    triples = _triples(15_000, 98)
    got = kernel_signs(triples)
    for i, (a, b, c) in enumerate(triples):
        want = _exact_sign(a, b, c)
        assert got[i, 0] == want, (i, got[i, 0], want)
        assert got[i, 1] == exact.orient(a, b, c, sos=True), i
        if want != 0:
            assert got[i, 1] == want, i
