// local_frame.cuh - the FP32 crossing tests in a leaf's local frame.
//
// The crossing tests of the exact query need the signs of
//   s2 = det[A; B; q] = q . (A x B),  s3 = det[R; q; A] = q . (A x R),
//   s4 = det[R; q; B] = q . (B x R)
// on the canonical FP64 XYZ of the query q, the leaf center R and the edge
// (A, B).  Evaluating them on an FP32 copy of q bounds the error by FP32's
// resolution on the unit sphere (~1e-7 rad), so every point closer than that
// to an edge escalates.  Here the offset d = q - R is computed in FP32 from
// the differences of the canonical radians (sum-to-product identities with
// accurate sines of the half differences), so its error is relative to |d|,
// about the leaf's size, and
//   s2 = sign(R.(A x B) + d.(A x B)),  s3 = sign(d.(A x R)),  s4 = sign(d.(B x R))
// since R.(A x R) = R.(B x R) = 0.  R.(A x B) and the three cross products
// are stored per (leaf, edge) record, each rounded from a value within a few
// FP64 ulp of the exact one.
//
// Error bound (u = 2^-24).  With h = half the canonical differences, m the
// midpoints reduced to [-pi, pi]: |fl(m) - m| <= u pi; sinf/cosf are within
// 2 ulp (CUDA's documented bound; the host functions are tighter), so each
// of sin/cos(m) and of sin(a), cos(a), cos(b0) is within 7.2e-7 absolutely,
// sin(h) within 3u relatively; each component of d is then within
// KAPPA * (|hA| + |hB|) + DELTA of the offset of the canonical points
// (worst case about 2e-6 * (|hA| + |hB|)), where DELTA covers the FP64
// rounding of the radian differences (up to +-2 pi wraps, about 6e-15) and
// the canonical conversion's own errors.  A dot product
// with float vectors each rounded from a value within a few FP64 ulp adds
// REL * (sum of |terms|).  The constants carry a margin of two or more.
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

struct Offset {
    float d[3];
    float err;  // bound on |d_i - (q - R)_i| for each component
};

// q from (lon, lat) and R from (lonR, latR), degrees, as the canonical
// conversion takes them (lat is the query's FakeLL latitude).  False when the
// offset is not small (|half differences| above ~0.5 rad): the caller defers.
LFHD bool offset(double lon, double lat, double lonR, double latR, Offset& o)
{
    const double a = gahhg_canon_rad(lon), a0 = gahhg_canon_rad(lonR);
    const double b = gahhg_canon_rad(lat), b0 = gahhg_canon_rad(latR);
    double ta = a - a0;
    const double k = rint(ta / TWO_PI_HI);
    ta = (ta - k * TWO_PI_HI) - k * TWO_PI_LO;
    const double ha = 0.5 * ta, hb = 0.5 * (b - b0);
    if (!(fabs(ha) < 0.5 && fabs(hb) < 0.5)) return false;
    double ma = a0 + ha;
    ma -= TWO_PI_HI * rint(ma / TWO_PI_HI);
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
    return true;
}

LFHD int sign_bounded(float v, float bound) { return v > bound ? 1 : (v < -bound ? -1 : 0); }

// sign(h + d . n), 0 when undecided (h = 0 for s3 and s4).
LFHD int sign_at(const Offset& o, const float* n, float h)
{
    const float t0 = o.d[0] * n[0], t1 = o.d[1] * n[1], t2 = o.d[2] * n[2];
    const float v = h + t0 + t1 + t2;
    const float bound = o.err * (fabsf(n[0]) + fabsf(n[1]) + fabsf(n[2])) +
                        REL * (fabsf(h) + fabsf(t0) + fabsf(t1) + fabsf(t2)) + 1e-30f;
    return sign_bounded(v, bound);
}

}  // namespace local_frame
}  // namespace gahhg
