/*
 * gahhg_canon.h - canonical lon/lat -> unit-vector conversion.
 *
 * Every label this library produces is a function of the FP64 XYZ vectors of
 * the polygon vertices and query points.  The reference converts on the host
 * with the platform libm (source/GPISPPolygon.cuh:21-30 LLVertex::LL2XYZ and
 * :82-92 FakeLLVertex::FakeLL2XYZ), so its bits depend on the C runtime.  To
 * make host, device and test oracles agree bit for bit, the conversion here
 * uses one sine/cosine written from first principles:
 *
 *   - Cody-Waite argument reduction by pi/2 with a three-part split of pi/2
 *     (the split is the binary expansion of pi/2, computed with exact rational
 *     arithmetic), fused multiply-adds for the reduction;
 *   - the Taylor series of sin and cos (coefficients 1/n! rounded to double)
 *     on |r| <= pi/4, evaluated by Horner's rule with explicit fma().
 *
 * Only explicit fma() calls are fused; every other operation is a separately
 * rounded IEEE-754 double operation, so a compiler that does not contract
 * (gcc -ffp-contract=off, nvcc --fmad=false) yields identical bits on the CPU
 * and on the GPU.  Accuracy is about 1 ulp, which the tests check against a
 * high-precision reference.
 *
 * The degree->radian step keeps the reference's truncated PI
 * (source/GPISPDS.cuh:7 `#define PI 3.14159265`) and its evaluation order
 * `deg * PI / 180.0`.
 */
#ifndef GAHHG_CANON_H
#define GAHHG_CANON_H

#include <math.h>

#if defined(__CUDACC__)
#define GAHHG_HD __host__ __device__ __forceinline__
#else
#define GAHHG_HD static inline
#endif

#ifdef __cplusplus
extern "C++" {
#endif

/* Truncated PI used by every reference conversion (source/GPISPDS.cuh:7). */
#define GAHHG_PI_TRUNC 3.14159265

/* pi/2 = P1 + P2 + P3 (exact binary split, |P3| ~ 1.5e-33). */
#define GAHHG_PIO2_1 1.5707963267948966
#define GAHHG_PIO2_2 6.123233995736766e-17
#define GAHHG_PIO2_3 (-1.4973849048591698e-33)
#define GAHHG_2_OVER_PI 0.6366197723675814

/* Sine and cosine of x (radians). */
GAHHG_HD void gahhg_canon_sincos(double x, double* s_out, double* c_out)
{
    double kf = nearbyint(x * GAHHG_2_OVER_PI);
    double r = fma(-kf, GAHHG_PIO2_1, x);
    r = fma(-kf, GAHHG_PIO2_2, r);
    r = fma(-kf, GAHHG_PIO2_3, r);
    double r2 = r * r;

    /* sin(r) = r + r^3 * (-1/3! + r^2 (1/5! - r^2 (1/7! - ... 1/17!))) */
    double ps = 2.8114572543455206e-15;          /*  1/17! */
    ps = fma(ps, r2, -7.647163731819816e-13);    /* -1/15! */
    ps = fma(ps, r2, 1.6059043836821613e-10);    /*  1/13! */
    ps = fma(ps, r2, -2.505210838544172e-08);    /* -1/11! */
    ps = fma(ps, r2, 2.7557319223985893e-06);    /*  1/9!  */
    ps = fma(ps, r2, -0.0001984126984126984);    /* -1/7!  */
    ps = fma(ps, r2, 0.008333333333333333);      /*  1/5!  */
    ps = fma(ps, r2, -0.16666666666666666);      /* -1/3!  */
    double s = fma(r * r2, ps, r);

    /* cos(r) = 1 + r^2 * (-1/2! + r^2 (1/4! - r^2 (1/6! - ... 1/18!))) */
    double pc = -1.5619206968586225e-16;         /* -1/18! */
    pc = fma(pc, r2, 4.779477332387385e-14);     /*  1/16! */
    pc = fma(pc, r2, -1.1470745597729725e-11);   /* -1/14! */
    pc = fma(pc, r2, 2.08767569878681e-09);      /*  1/12! */
    pc = fma(pc, r2, -2.755731922398589e-07);    /* -1/10! */
    pc = fma(pc, r2, 2.48015873015873e-05);      /*  1/8!  */
    pc = fma(pc, r2, -0.001388888888888889);     /* -1/6!  */
    pc = fma(pc, r2, 0.041666666666666664);      /*  1/4!  */
    pc = fma(pc, r2, -0.5);                      /* -1/2!  */
    double c = fma(r2, pc, 1.0);

    long long q = (long long)kf & 3;
    double so, co;
    if (q == 0)      { so = s;  co = c;  }
    else if (q == 1) { so = c;  co = -s; }
    else if (q == 2) { so = -s; co = -c; }
    else             { so = -c; co = s;  }
    *s_out = so;
    *c_out = co;
}

/* Degrees -> radians exactly as the reference evaluates `deg * PI / 180.0`. */
GAHHG_HD double gahhg_canon_rad(double deg)
{
    return (deg * GAHHG_PI_TRUNC) / 180.0;
}

/* Polygon vertex: LLVertex::LL2XYZ (source/GPISPPolygon.cuh:21-30). */
GAHHG_HD void gahhg_canon_vertex_xyz(double lon, double lat, double* xyz)
{
    double sa, ca, so, co;
    gahhg_canon_sincos(gahhg_canon_rad(lat), &sa, &ca);
    gahhg_canon_sincos(gahhg_canon_rad(lon), &so, &co);
    xyz[0] = ca * so;
    xyz[1] = sa;
    xyz[2] = ca * co;
}

/* Latitude a query point is converted at: the reference routes query points
 * through FakeLLVertex (source/GPISPTP.cu:67-68, GPISPPolygon.cuh:72,82-85),
 * fakela = la + 90 and back, which rounds in FP64. */
GAHHG_HD double gahhg_canon_query_lat(double lat)
{
    double fakela = lat + 90.0;
    return fakela > 180.0 ? 270.0 - fakela : fakela - 90.0;
}

/* Query point: FakeLLVertex::FakeLL2XYZ (source/GPISPPolygon.cuh:82-92). */
GAHHG_HD void gahhg_canon_query_xyz(double lon, double lat, double* xyz)
{
    gahhg_canon_vertex_xyz(lon, gahhg_canon_query_lat(lat), xyz);
}

#ifdef __cplusplus
}
#endif

#endif /* GAHHG_CANON_H */
