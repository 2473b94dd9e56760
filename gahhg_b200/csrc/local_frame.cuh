// local_frame.cuh - the FP32 crossing tests in a leaf's local frame.
//
// The crossing tests of the exact query need the signs of
//   s2 = det[A; B; q],  s3 = det[R; q; A],  s4 = det[R; q; B]
// on the canonical FP64 XYZ of the query q, the leaf center R and the edge
// (A, B).  Evaluating them on an FP32 copy of q bounds the error by FP32's
// resolution on the unit sphere (~1e-7 rad), so every point closer than that
// to an edge would escalate.  Here the offset d = q - R is computed in FP32
// from the differences of the canonical radians (sum-to-product identities
// with accurate sines of the half differences), so its error is relative to
// |d|, about the leaf's size; the three determinants are then evaluated in
// the tangent frame of R (see edge_record below), where an edge is four
// floats and the query two coordinates and q . R.
//
// Error bound of the offset (u = 2^-24).  With h = half the canonical
// differences, m the midpoints reduced to [-pi, pi]: |fl(m) - m| <= u pi;
// sinf/cosf are within 2 ulp (CUDA's documented bound; the host functions are
// tighter), so each of sin/cos(m) and of sin(a), cos(a), cos(b0) is within
// 7.2e-7 absolutely, sin(h) within 3u relatively; each component of d is then
// within KAPPA * (|hA| + |hB|) + DELTA of the offset of the canonical points
// (worst case about 2e-6 * (|hA| + |hB|)), where DELTA covers the FP64
// rounding of the radian differences (up to +-2 pi wraps, about 6e-15) and
// the canonical conversion's own errors.  A product of floats each rounded
// from a value within a few FP64 ulp adds REL * (sum of |terms|).  The
// constants carry a margin of two or more.
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

constexpr float KAPPA = 8.0e-6f;   // per component of d, per radian of |hA| + |hB|
constexpr float DELTA = 3.0e-14f;  // absolute, per component of d
constexpr float REL = 1.0e-6f;     // relative, per term of a dot product (rounding of terms and sums)
constexpr double TWO_PI_HI = 6.283185307179586;          // 2 pi rounded to double
constexpr double TWO_PI_LO = 2.4492935982947064e-16;     // 2 pi - TWO_PI_HI
constexpr double INV_TWO_PI = 0.15915494309189535;       // 1 / (2 pi) rounded to double

struct Offset {
    float d[3];
    float err;             // bound on |d_i - (q - R)_i| for each component
    float cl, sl, cp, sp;  // cos/sin of R's longitude and latitude, each within BASIS_ERR
};

// q from (lon, lat) and R from (lonR, latR), degrees, as the canonical
// conversion takes them (lat is the query's FakeLL latitude).  False when the
// offset is not small (|half differences| above ~0.5 rad): the caller defers.
LFHD bool offset(double lon, double lat, double lonR, double latR, Offset& o)
{
    const double a = gahhg_canon_rad(lon), a0 = gahhg_canon_rad(lonR);
    const double b = gahhg_canon_rad(lat), b0 = gahhg_canon_rad(latR);
    // the nearest multiple of 2 pi by a reciprocal product: where it can differ
    // from the quotient's (a half-integer number of turns) |ha| ~ pi / 2, and
    // the offset is refused below; the midpoint lands in [-pi, pi] up to ulps
    double ta = a - a0;
    const double k = rint(ta * INV_TWO_PI);
    ta = (ta - k * TWO_PI_HI) - k * TWO_PI_LO;
    const double ha = 0.5 * ta, hb = 0.5 * (b - b0);
    if (!(fabs(ha) < 0.5 && fabs(hb) < 0.5)) return false;
    double ma = a0 + ha;
    ma -= TWO_PI_HI * rint(ma * INV_TWO_PI);
    const double mb = b0 + hb;
    const float fha = (float)ha, fhb = (float)hb, fma_ = (float)ma, fmb = (float)mb;
    const float sma = sinf(fma_), cma = cosf(fma_);
    const float smb = sinf(fmb), cmb = cosf(fmb);
    const float sha = sinf(fha), shb = sinf(fhb);
    const float cha = cosf(fha), chb = cosf(fhb);
    const float sin_a = sma * cha + cma * sha;  // a = ma + ha
    const float cos_a = cma * cha - sma * sha;
    const float cos_b0 = cmb * chb + smb * shb;  // b0 = mb - hb
    const float dc = -2.0f * smb * shb;          // cos b - cos b0
    const float dsa = 2.0f * cma * sha;          // sin a - sin a0
    const float dca = -2.0f * sma * sha;         // cos a - cos a0
    o.d[0] = dc * sin_a + cos_b0 * dsa;          // cos b sin a - cos b0 sin a0
    o.d[1] = 2.0f * cmb * shb;                   // sin b - sin b0
    o.d[2] = dc * cos_a + cos_b0 * dca;          // cos b cos a - cos b0 cos a0
    o.err = KAPPA * (fabsf(fha) + fabsf(fhb)) + DELTA;
    o.sl = sma * cha - cma * sha;  // a0 = ma - ha
    o.cl = cma * cha + sma * sha;
    o.sp = smb * chb - cmb * shb;  // b0 = mb - hb
    o.cp = cos_b0;
    return true;
}

LFHD int sign_bounded(float v, float bound) { return v > bound ? 1 : (v < -bound ? -1 : 0); }

// ---- the leaf's tangent frame -------------------------------------------
//
// With R at canonical radians (a0, b0), e1 = (cos a0, 0, -sin a0) (east) and
// e2 = (-sin b0 sin a0, cos b0, -sin b0 cos a0) (north) complete R to a
// right-handed orthonormal basis (det[R; e1; e2] = 1).  In it a point X has
// coordinates (X.R, X.e1, X.e2); an edge end A with A.R > 0 is stored as its
// gnomonic coordinates a = (A.e1, A.e2) / (A.R), and the query as
// w = q.R = 1 + d.R and p = (d.e1, d.e2) (R.e1 = R.e2 = 0).  Then, exactly,
//   det[A; B; q] = (A.R)(B.R) (w (a1 b2 - a2 b1) + (b1 - a1) p2 - (b2 - a2) p1)
//   det[R; q; A] = (A.R) (p1 a2 - p2 a1)
// (rows expanded in the basis), so an edge needs four floats.  Records are
// stored in the order that makes orient(A, B, R) = +1; swapping A and B
// negates det[A; B; q] and exchanges the two end tests, and the crossing test
// (s2 != s1, s3 == s2, s4 == -s2) is symmetric under that exchange.
//
// Error terms beyond the offset's: the basis computed in FP32 from the sines
// and cosines of the offset (BASIS_ERR absolutely per component) perturbs p
// and w by BASIS_ERR (|d0| + |d1| + |d2|) each, three times over; the stored
// coordinates are rounded from FP64 values within ~1e-16 relatively (REL per
// product covers them and the FP32 arithmetic); R's canonical FP64 point
// differs from the exact one at (a0, b0) by ~1e-16, which adds at most
// 1e-16 (|p| + |a|) to an end test (END_DELTA, with a large margin) and is
// inside the offset's DELTA for p and w.
constexpr float BASIS_ERR = 2.0e-6f;
constexpr float END_DELTA = 1.0e-14f;

struct Frame {
    float p1, p2, w;
    float errp, errw;  // bounds on |p_i - exact| and |w - exact|
};

LFHD void project(const Offset& o, Frame& f)
{
    const float t = o.d[0] * o.sl + o.d[2] * o.cl;
    f.p1 = o.d[0] * o.cl - o.d[2] * o.sl;
    f.p2 = o.d[1] * o.cp - o.sp * t;
    f.w = 1.0f + (o.cp * t + o.sp * o.d[1]);
    const float dn = fabsf(o.d[0]) + fabsf(o.d[1]) + fabsf(o.d[2]);
    f.errp = 2.0f * o.err + (3.0f * BASIS_ERR + REL) * dn;
    f.errw = f.errp + 1.0e-7f;
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

// sign det[A; B; q] for a record (a1, a2, b1, b2) in its stored order.
LFHD int sign_edge(const Frame& f, float a1, float a2, float b1, float b2)
{
    const float u1 = b1 - a1, u2 = b2 - a2;
    const float c = a1 * b2 - a2 * b1;
    const float v = f.w * c + (u1 * f.p2 - u2 * f.p1);
    const float bound = f.errp * (fabsf(u1) + fabsf(u2)) + f.errw * fabsf(c) +
                        REL * (fabsf(f.w) * (fabsf(a1 * b2) + fabsf(a2 * b1)) + (fabsf(a1) + fabsf(b1)) * fabsf(f.p2) +
                               (fabsf(a2) + fabsf(b2)) * fabsf(f.p1)) +
                        1e-30f;
    return sign_bounded(v, bound);
}

// sign det[R; q; X] for an end (x1, x2) of a record.
LFHD int sign_end(const Frame& f, float x1, float x2)
{
    const float v = f.p1 * x2 - f.p2 * x1;
    const float bound = f.errp * (fabsf(x1) + fabsf(x2)) + REL * (fabsf(f.p1 * x2) + fabsf(f.p2 * x1)) +
                        END_DELTA * (fabsf(x1) + fabsf(x2) + fabsf(f.p1) + fabsf(f.p2)) + 1e-30f;
    return sign_bounded(v, bound);
}

}  // namespace local_frame
}  // namespace gahhg
