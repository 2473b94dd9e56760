// local_frame.cuh - the FP32 crossing tests in a leaf's local frame.
//
// The crossing tests of the exact query need the signs of
//   s2 = det[A; B; q],  s3 = det[R; q; A],  s4 = det[R; q; B]
// on the canonical FP64 XYZ of the query q, the leaf center R and the edge
// (A, B).  Evaluating them on an FP32 copy of q bounds the error by FP32's
// resolution on the unit sphere (~1e-7 rad), so every point closer than that
// to an edge would escalate.  Here q is expressed in the tangent frame of R
// (see edge_record below) directly from the angle differences to R, so the
// error of its frame coordinates is relative to their size (about the leaf's
// size); an edge is four floats in the same frame.
//
// The frame coordinates (frame_at).  With canonical radians (a, b) of q and
// (a0, b0) of R, dl = a - a0 (reduced by 2 pi), dp = b - b0 and phi = b:
//   p1 = q.e1 = cos phi sin dl
//   p2 = q.e2 = sin dp + sin b0 cos phi (1 - cos dl)
//   w  = q.R  = cos dp - cos b0 cos phi (1 - cos dl)
//   cos phi   = cos b0 cos dp - sin b0 sin dp
// The differences dl, dp come from the degree differences in FP64 (one
// multiplication by pi'/180, no division), so they carry an absolute error
// E_RAD against the canonical radians' difference besides their rounding to
// FP32.  sin, cos and 1 - cos of |x| <= 0.5 are Taylor polynomials in FP32
// (coefficients 1/n! rounded to float, Horner's rule with explicit fmaf,
// truncated where the next term is below 1e-11 relative).  sin b0 and cos b0
// are stored per leaf (FP64 canonical values rounded to float).  Every step
// is one or two FP32 roundings, and frame_at evaluates, per point, a bound on
// each coordinate's error from the magnitudes it computed (the derivation is
// beside the code); the bound is doubled to cover its own FP32 evaluation and
// the second-order terms left out.
//
// Only explicit fmaf() calls fuse (nvcc --fmad=false, host -ffp-contract=off),
// so the host build of this header that the soundness tests run gives the
// device's bits.
#pragma once

#include <math.h>

#include "gahhg_canon.h"

#ifdef __CUDACC__
#define LFHD __host__ __device__ __forceinline__
#else
#define LFHD inline
#endif

namespace gahhg {
namespace local_frame {

constexpr float EPS = 5.9604645e-8f;                      // 2^-24, FP32 unit roundoff
constexpr double RAD_PER_DEG = GAHHG_PI_TRUNC / 180.0;    // the canonical conversion's pi' / 180, rounded
constexpr double TWO_PI_HI = 6.283185307179586;          // 2 pi rounded to double
constexpr double TWO_PI_LO = 2.4492935982947064e-16;     // 2 pi - TWO_PI_HI
constexpr double INV_TWO_PI = 0.15915494309189535;       // 1 / (2 pi) rounded to double
// Absolute error of the FP64 differences against the canonical radians'
// difference, for |lon|, |lonR| <= 540 deg: each canonical radian value is
// within 2 ulp of x pi' / 180 (|a| <= 9.43: 4.2e-15 for both), the
// difference and product add 3 ulp of the result, the reduction by 2 pi
// (|k| <= 3, two-part constant) about 4e-15; 1.1e-14 in all, 3e-14 here.
constexpr float E_RAD = 3.0e-14f;
// Absolute floor added to each coordinate's bound: the canonical XYZ of q
// and R differ from the exact sine/cosine points at their canonical radians
// by a few 1e-16 per component, which moves each determinant by at most that
// times the norm of the other rows' cross product.
constexpr float DELTA = 3.0e-14f;
// Relative error per term of the determinants in sign_edge / sign_end: the
// records' rounding to float (2 eps per coordinate product) and the fmaf
// evaluation (4 eps for sign_edge, 2 for sign_end); 10 eps here.
constexpr float REL = 6.0e-7f;

// Taylor polynomials for |x| <= 0.5 (FP32, explicit fmaf).
//   taylor_sin: |S - sin x| <= 2 eps |x|   (x^3 term: x3 rounded twice, P within 1.1 eps)
//   taylor_vers: 1 - cos x, |H - (1 - cos x)| <= 5 eps H
LFHD float taylor_sin(float x)
{
    const float x2 = x * x;
    float p = fmaf(x2, 2.7557319e-6f, -1.9841270e-4f);  //  1/9!, -1/7!
    p = fmaf(p, x2, 8.3333333e-3f);                      //  1/5!
    p = fmaf(p, x2, -1.6666667e-1f);                     // -1/3!
    return fmaf(x * x2, p, x);
}

LFHD float taylor_vers(float x)
{
    const float x2 = x * x;
    float p = fmaf(x2, 2.7557319e-7f, -2.4801587e-5f);  //  1/10!, -1/8!
    p = fmaf(p, x2, 1.3888889e-3f);                      //  1/6!
    p = fmaf(p, x2, -4.1666667e-2f);                     // -1/4!
    p = fmaf(p, x2, 0.5f);                               //  1/2!
    return x2 * p;
}

// The query's coordinates in the leaf's frame and bounds on their errors:
// |p_i - exact| <= errp, |w - exact| <= errw.
struct Frame {
    float p1, p2, w;
    float errp, errw;
};

// q at (lon, lat) degrees (lat: the query's FakeLL latitude, as the canonical
// conversion takes it), the leaf center at (lonR, latR) degrees with sb, cb =
// sin and cos of its canonical latitude rounded to float.  False when an
// angle difference exceeds 0.5 rad (the caller defers to FP64); then q.R >=
// cos 0.5 - (1 - cos 0.5) > 0.75.
LFHD bool frame_at(double lon, double lat, double lonR, double latR, float sb, float cb, Frame& f)
{
    double dl = (lon - lonR) * RAD_PER_DEG;
    const double k = rint(dl * INV_TWO_PI);
    dl = (dl - k * TWO_PI_HI) - k * TWO_PI_LO;
    const double dp = (lat - latR) * RAD_PER_DEG;
    if (!(fabs(dl) <= 0.5 && fabs(dp) <= 0.5)) return false;
    const float xl = (float)dl, xp = (float)dp;
    const float axl = fabsf(xl), axp = fabsf(xp);
    // input errors against the canonical differences: rounding to float and E_RAD
    const float etal = fmaf(axl, 1.0000001f * EPS, E_RAD), etap = fmaf(axp, 1.0000001f * EPS, E_RAD);
    const float sp = taylor_sin(xp), hp = taylor_vers(xp), cp = 1.0f - hp;
    const float sl = taylor_sin(xl), hl = taylor_vers(xl);
    // cos phi = cos b0 cos dp - sin b0 sin dp
    const float m1 = sb * sp;
    const float cf = fmaf(cb, cp, -m1);
    const float t = cf * hl;  // cos phi (1 - cos dl)
    f.p1 = cf * sl;
    f.p2 = fmaf(sb, t, sp);
    f.w = fmaf(-cb, t, cp);
    // Error bounds (first order; |sb|, |cb| <= 1, |xl|, |xp| <= 0.5):
    //  es_p = |sp - sin dp| <= 2 eps |xp| + etap     (sin is 1-Lipschitz)
    //  ec_p = |cp - cos dp| <= 2 eps + |xp| etap     (1 - hp: one rounding, 5 eps hp <= 0.62 eps)
    //  es_l = |sl - sin dl| <= 2 eps |xl| + etal
    //  eh_l = |hl - (1 - cos dl)| <= 5 eps hl + |xl| etal
    //  stored sb, cb: within eps |.| + 3e-16 of sin b0, cos b0
    //  E_cf = |cf - cos phi| <= eps |cf| + eps |m1| + (eps |cb| + |cb| ec_p) + (eps |sb sp| + |sb| es_p)
    //       <= eps (|cf| + 2 |m1| + 3 |cb| + 2 |xp|) + 1.5 etap + 1e-15
    //  |p1 - p1*| <= eps |p1| + E_cf |sl| + |cf| es_l
    //  |t - t*|   <= eps |t| + E_cf hl + |cf| eh_l
    //  |p2 - p2*| <= eps |p2| + eps |t| + |t - t*| + es_p
    //  |w - w*|   <= eps |w| + ec_p + eps |t| + |t - t*|
    const float acf = fabsf(cf), at = fabsf(t);
    const float ecf = fmaf(EPS, acf + 2.0f * fabsf(m1) + 3.0f * fabsf(cb) + 2.0f * axp, fmaf(1.5f, etap, 1.0e-15f));
    const float ep1 = EPS * fabsf(f.p1) + ecf * fabsf(sl) + acf * fmaf(2.0f * EPS, axl, etal);
    const float et = EPS * at + ecf * hl + acf * fmaf(5.0f * EPS, hl, axl * etal);
    const float ep2 = EPS * (fabsf(f.p2) + at) + et + fmaf(2.0f * EPS, axp, etap);
    const float ew = EPS * (fabsf(f.w) + at) + et + fmaf(axp, etap, 2.0f * EPS);
    f.errp = fmaf(2.0f, fmaxf(ep1, ep2), DELTA);
    f.errw = fmaf(2.0f, ew, DELTA);
    return true;
}

// The tangent frame at the center (canonical radians of its degrees), FP64.
struct Basis {
    double e1[3], e2[3], R[3];
};

LFHD void basis_at(double lonR, double latR, Basis& f)
{
    const double a0 = gahhg_canon_rad(lonR), b0 = gahhg_canon_rad(latR);
    const double sa = sin(a0), ca = cos(a0), sb = sin(b0), cb = cos(b0);
    f.e1[0] = ca;
    f.e1[1] = 0.0;
    f.e1[2] = -sa;
    f.e2[0] = -sb * sa;
    f.e2[1] = cb;
    f.e2[2] = -sb * ca;
    f.R[0] = cb * sa;
    f.R[1] = sb;
    f.R[2] = cb * ca;
}

// Gnomonic coordinates of A, B in the frame f on FP64 points, rounded to
// float; r gets (a1, a2, b1, b2), in the order swap ? (B, A) : (A, B).  An end
// with X.R < 0.5 gives NaN coordinates (every test on the record is
// undecided).
LFHD void edge_record(const double* A, const double* B, const Basis& f, bool swap, float* r)
{
    const double* X[2] = {swap ? B : A, swap ? A : B};
    for (int k = 0; k < 2; k++) {
        const double* x = X[k];
        const double den = x[0] * f.R[0] + x[1] * f.R[1] + x[2] * f.R[2];
        if (!(den >= 0.5)) {
            r[2 * k] = r[2 * k + 1] = NAN;
            continue;
        }
        r[2 * k] = (float)((x[0] * f.e1[0] + x[2] * f.e1[2]) / den);
        r[2 * k + 1] = (float)((x[0] * f.e2[0] + x[1] * f.e2[1] + x[2] * f.e2[2]) / den);
    }
}

// Canonical R against the exact frame point: at most a few 1e-16 per
// component, which moves det[R; q; X] / (X.R) by about that times
// |p1| + |p2| + |x1| + |x2|; END_DELTA carries a margin above 30.
constexpr float END_DELTA = 1.0e-14f;

// The record tests' per-point constants.  For a record (a1, a2, b1, b2) with
// T = |a1| + |a2| + |b1| + |b2|:
//   s2 = sign det[A; B; q]: v2 = w c + (b1 - a1) p2 - (b2 - a2) p1,
//        c = a1 b2 - a2 b1 = fl(a1 b2 - m), m = fl(a2 b1).  Its error is the
//        frame's, errp (|u1| + |u2|) + errw |c|, plus REL times
//        S = |w| (|a1 b2| + |a2 b1|) + (|a1| + |b1|) |p2| + (|a2| + |b2|) |p1|;
//        with |u1| + |u2| <= T, |a1 b2| + |a2 b1| <= |c| + 2 |m| and
//        S <= |w| (|c| + 2 |m|) + max(|p1|, |p2|) T (each up to a rounding,
//        inside REL's margin) it is at most K1 T + K2 |c| + K3 |m|.
//   s3 = sign det[R; q; A]: v3 = p1 a2 - p2 a1, error at most
//        errp (|a1| + |a2|) + REL (|p1 a2| + |p2 a1|) + END_DELTA (|a1| + |a2| + |p1| + |p2|)
//        <= KE (|a1| + |a2|) + DE; s4 likewise for B.
struct Tests {
    float p1, p2, w;
    float K1, K2, K3;  // s2 bound: K1 T + K2 |c| + K3 |m|
    float KE, DE;      // end bound: KE (|x1| + |x2|) + DE
};

LFHD void tests_of(const Frame& f, Tests& t)
{
    const float P = fmaxf(fabsf(f.p1), fabsf(f.p2)), P1 = fabsf(f.p1) + fabsf(f.p2), aw = fabsf(f.w);
    t.p1 = f.p1;
    t.p2 = f.p2;
    t.w = f.w;
    t.K1 = fmaf(REL, P, f.errp);
    t.K2 = fmaf(REL, aw, f.errw);
    t.K3 = 2.0f * REL * aw;
    t.KE = fmaf(REL, P1, f.errp + END_DELTA);
    t.DE = fmaf(END_DELTA, P1, 1e-30f);
}

LFHD int sign_bounded(float v, float bound) { return v > bound ? 1 : (v < -bound ? -1 : 0); }

// sign det[A; B; q] for a record (a1, a2, b1, b2) in its stored order.
LFHD int sign_edge(const Tests& t, float a1, float a2, float b1, float b2)
{
    const float u1 = b1 - a1, u2 = b2 - a2;
    const float m = a2 * b1;
    const float c = fmaf(a1, b2, -m);
    const float v = fmaf(t.w, c, fmaf(u1, t.p2, -(u2 * t.p1)));
    const float T = (fabsf(a1) + fabsf(a2)) + (fabsf(b1) + fabsf(b2));
    return sign_bounded(v, fmaf(t.K1, T, fmaf(t.K2, fabsf(c), t.K3 * fabsf(m))));
}

// sign det[R; q; X] for an end (x1, x2) of a record.
LFHD int sign_end(const Tests& t, float x1, float x2)
{
    const float v = fmaf(t.p1, x2, -(t.p2 * x1));
    return sign_bounded(v, fmaf(t.KE, fabsf(x1) + fabsf(x2), t.DE));
}

// The crossing test of one record in its stored order (orient(A, B, R) = +1):
// arc(R, q) crosses the edge when s2 = -1, s3 = -1 and s4 = +1.  Returns 1
// (crossing), 0 (none: some sign rules it out, decided even when another is
// not) or -1 (undecided).  All three signs are evaluated without branches,
// with the bounds of sign_edge / sign_end.
LFHD int record_crossing(const Tests& t, float a1, float a2, float b1, float b2)
{
    const float v3 = fmaf(t.p1, a2, -(t.p2 * a1));
    const float v4 = fmaf(t.p1, b2, -(t.p2 * b1));
    const float na = fabsf(a1) + fabsf(a2), nb = fabsf(b1) + fabsf(b2);
    const float B3 = fmaf(t.KE, na, t.DE), B4 = fmaf(t.KE, nb, t.DE);
    const float u1 = b1 - a1, u2 = b2 - a2;
    const float m = a2 * b1;
    const float c = fmaf(a1, b2, -m);
    const float v2 = fmaf(t.w, c, fmaf(u1, t.p2, -(u2 * t.p1)));
    const float B2 = fmaf(t.K1, na + nb, fmaf(t.K2, fabsf(c), t.K3 * fabsf(m)));
    const bool none = (v2 > B2) | (v3 > B3) | (v4 < -B4);
    const bool cross = (v2 < -B2) & (v3 < -B3) & (v4 > B4);
    return cross ? 1 : (none ? 0 : -1);
}

}  // namespace local_frame
}  // namespace gahhg
