// exact_pred.cuh - exact orientation predicates for the exact-label engine.
//
// orient(a,b,c) = sign(det[a;b;c]) = sign(a . (b x c)) on FP64 coordinates,
// decided in three stages (the query kernel adds an FP32 stage in front):
//   1. FP64 evaluation with the forward error bound 8 eps |permanent|;
//   2. exact summation of the 24 error-free triple products with
//      floating-point expansions (two_sum / two_product, Shewchuk 1997);
//   3. for an exactly vanishing determinant, simulation of simplicity
//      (Edelsbrunner & Muecke 1990): rows ranked lexicographically, entry
//      (r, c) perturbed by eps^(2^(3r+c)), sign of the first non-vanishing
//      coefficient of det(M + E) in increasing order of exponent.
// Identical points are not separated (the function returns 0); callers
// exclude them.  All functions are host+device; no fused multiply-add except
// the explicit fma() of two_prod (sources compile with --fmad=false).
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define XHD __host__ __device__ __forceinline__
#define XHDN __host__ __device__ __noinline__
#else
#define XHD inline
#define XHDN inline
#endif

namespace gahhg {
namespace exact {

constexpr double EPS53 = 1.1102230246251565e-16;  // 2^-53

XHD void two_sum(double a, double b, double& s, double& e)
{
    double x = a + b;
    double bv = x - a;
    double av = x - bv;
    s = x;
    e = (a - av) + (b - bv);
}

XHD void two_prod(double a, double b, double& p, double& e)
{
    p = a * b;
    e = fma(a, b, -p);
}

// Exact sign of the sum of n exactly representable terms (n <= 24).
XHDN int sum_sign(const double* t, int n)
{
    double e[48];
    int m = 0;
    for (int i = 0; i < n; i++) {
        double q = t[i];
        if (q == 0.0) continue;
        int k = 0;
        for (int j = 0; j < m; j++) {
            double s, r;
            two_sum(q, e[j], s, r);
            if (r != 0.0) e[k++] = r;
            q = s;
        }
        if (q != 0.0 || k == 0) e[k++] = q;
        m = k;
    }
    for (int i = m - 1; i >= 0; i--) {
        if (e[i] > 0) return 1;
        if (e[i] < 0) return -1;
    }
    return 0;
}

// The sum of n exactly representable terms (n <= 24) to within a few ulp of
// the exact sum: the terms are accumulated into a non-overlapping expansion
// (as in sum_sign), whose components are then added from the smallest up.
XHDN double sum_value(const double* t, int n)
{
    double e[48];
    int m = 0;
    for (int i = 0; i < n; i++) {
        double q = t[i];
        if (q == 0.0) continue;
        int k = 0;
        for (int j = 0; j < m; j++) {
            double s, r;
            two_sum(q, e[j], s, r);
            if (r != 0.0) e[k++] = r;
            q = s;
        }
        if (q != 0.0 || k == 0) e[k++] = q;
        m = k;
    }
    double v = 0.0;
    for (int i = 0; i < m; i++) v += e[i];
    return v;
}

// u0 v1 - u1 v0 to within a few ulp (exact products, then sum_value).
XHD double det2_value(double u0, double u1, double v0, double v1)
{
    double t[4];
    two_prod(u0, v1, t[0], t[1]);
    two_prod(-u1, v0, t[2], t[3]);
    return sum_value(t, 4);
}

XHD void triple(double a, double b, double c, double* o)
{
    double p, e;
    two_prod(b, c, p, e);
    two_prod(a, p, o[0], o[1]);
    two_prod(a, e, o[2], o[3]);
}

XHDN int det3_sign(const double* a, const double* b, const double* c)
{
    double t[24];
    triple(a[0], b[1], c[2], t + 0);
    triple(-a[0], b[2], c[1], t + 4);
    triple(a[1], b[2], c[0], t + 8);
    triple(-a[1], b[0], c[2], t + 12);
    triple(a[2], b[0], c[1], t + 16);
    triple(-a[2], b[1], c[0], t + 20);
    return sum_sign(t, 24);
}

// det[a; b; c] to within a few ulp of its exact value.
XHDN double det3_value(const double* a, const double* b, const double* c)
{
    double t[24];
    triple(a[0], b[1], c[2], t + 0);
    triple(-a[0], b[2], c[1], t + 4);
    triple(a[1], b[2], c[0], t + 8);
    triple(-a[1], b[0], c[2], t + 12);
    triple(a[2], b[0], c[1], t + 16);
    triple(-a[2], b[1], c[0], t + 20);
    return sum_value(t, 24);
}

// a x b, each component to within a few ulp.
XHD void cross_value(const double* a, const double* b, double* o)
{
    o[0] = det2_value(a[1], a[2], b[1], b[2]);
    o[1] = det2_value(a[2], a[0], b[2], b[0]);
    o[2] = det2_value(a[0], a[1], b[0], b[1]);
}

XHD int det2_sign(double u0, double u1, double v0, double v1)
{
    double t[4];
    two_prod(u0, v1, t[0], t[1]);
    two_prod(-u1, v0, t[2], t[3]);
    return sum_sign(t, 4);
}

XHD bool same(const double* p, const double* q) { return p[0] == q[0] && p[1] == q[1] && p[2] == q[2]; }

XHD bool lex_less(const double* p, const double* q)
{
    if (p[0] != q[0]) return p[0] < q[0];
    if (p[1] != q[1]) return p[1] < q[1];
    return p[2] < q[2];
}

XHD int fsign(double x) { return (x > 0) - (x < 0); }

// Symbolic perturbation of an exactly singular det[a;b;c].
XHDN int sos_sign(const double* a, const double* b, const double* c)
{
    const double* P[3] = {a, b, c};
    int flip = 0;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2 - i; j++)
            if (lex_less(P[j + 1], P[j])) {
                const double* t = P[j];
                P[j] = P[j + 1];
                P[j + 1] = t;
                flip ^= 1;
            }
    if (same(P[0], P[1]) || same(P[1], P[2])) return 0;
    // permutations of {0,1,2} as col[row], with their signs
    const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    const int psg[6] = {1, -1, -1, 1, 1, -1};
    for (int mask = 1; mask < 512; mask++) {
        int rows = 0, cols = 0, cnt = 0;
        int er[3], ec[3];
        bool ok = true;
        for (int p = 0; p < 9; p++) {
            if (!((mask >> p) & 1)) continue;
            const int r = p / 3, c = p % 3;
            if (((rows >> r) & 1) || ((cols >> c) & 1) || cnt == 3) {
                ok = false;
                break;
            }
            rows |= 1 << r;
            cols |= 1 << c;
            er[cnt] = r;
            ec[cnt] = c;
            cnt++;
        }
        if (!ok) continue;
        int s = 0;
        if (cnt == 1) {
            const int r = er[0], c = ec[0];
            const int r0 = r == 0 ? 1 : 0, r1 = r == 2 ? 1 : 2;
            const int c0 = c == 0 ? 1 : 0, c1 = c == 2 ? 1 : 2;
            s = det2_sign(P[r0][c0], P[r0][c1], P[r1][c0], P[r1][c1]);
            if ((r + c) & 1) s = -s;
        } else {
            for (int k = 0; k < 6; k++) {
                bool match = true;
                for (int e = 0; e < cnt; e++)
                    if (perm[k][er[e]] != ec[e]) match = false;
                if (!match) continue;
                if (cnt == 3) {
                    s = psg[k];
                } else {
                    const int r3 = 3 - er[0] - er[1];
                    s = psg[k] * fsign(P[r3][perm[k][r3]]);
                }
                break;
            }
        }
        if (s != 0) return flip ? -s : s;
    }
    return 0;
}

// Stage 1 only: +-1 when the FP64 value is certain, 0 when it is not.
XHD int orient_fp64(const double* a, const double* b, const double* c)
{
    const double m0 = b[1] * c[2] - b[2] * c[1];
    const double m1 = b[2] * c[0] - b[0] * c[2];
    const double m2 = b[0] * c[1] - b[1] * c[0];
    const double d = a[0] * m0 + a[1] * m1 + a[2] * m2;
    const double perm = fabs(a[0]) * (fabs(b[1] * c[2]) + fabs(b[2] * c[1])) +
                        fabs(a[1]) * (fabs(b[2] * c[0]) + fabs(b[0] * c[2])) +
                        fabs(a[2]) * (fabs(b[0] * c[1]) + fabs(b[1] * c[0]));
    const double bound = 8.0 * EPS53 * perm;
    if (d > bound) return 1;
    if (d < -bound) return -1;
    return 0;
}

// Stage 1 for b and c close to a: det[a; b; c] = det[a; b - a; c - a] (row
// operations leave the determinant unchanged), evaluated on the rounded
// differences.  This is Shewchuk's orient3d(O, b, c, a) stage A up to sign:
// its bound (7 + 56 eps) eps x permanent(rows) covers the rounding of the
// differences, and the permanent shrinks with |b - a| |c - a|, so points far
// closer to an edge than orient_fp64 can resolve are still decided.
XHD int orient_fp64_near(const double* a, const double* b, const double* c)
{
    const double ux = b[0] - a[0], uy = b[1] - a[1], uz = b[2] - a[2];
    const double vx = c[0] - a[0], vy = c[1] - a[1], vz = c[2] - a[2];
    const double m0 = uy * vz - uz * vy;
    const double m1 = uz * vx - ux * vz;
    const double m2 = ux * vy - uy * vx;
    const double d = a[0] * m0 + a[1] * m1 + a[2] * m2;
    const double perm = fabs(a[0]) * (fabs(uy * vz) + fabs(uz * vy)) + fabs(a[1]) * (fabs(uz * vx) + fabs(ux * vz)) +
                        fabs(a[2]) * (fabs(ux * vy) + fabs(uy * vx));
    const double bound = (7.0 + 56.0 * EPS53) * EPS53 * perm;
    if (d > bound) return 1;
    if (d < -bound) return -1;
    return 0;
}

// Stages 2 and 3.
XHDN int orient_exact(const double* a, const double* b, const double* c)
{
    int s = det3_sign(a, b, c);
    if (s != 0) return s;
    return sos_sign(a, b, c);
}

XHD int orient(const double* a, const double* b, const double* c)
{
    int s = orient_fp64(a, b, c);
    if (s != 0) return s;
    return orient_exact(a, b, c);
}

// Arcs (r,q) and (a,b) cross: orient(a,r,b) = orient(b,q,a) = orient(r,b,q) =
// orient(q,a,r).  The four points must be pairwise distinct.
XHD bool crossing(const double* r, const double* q, const double* a, const double* b)
{
    const int acb = -orient(a, b, r);
    const int bda = orient(a, b, q);
    if (bda != acb) return false;
    const int cbd = -orient(r, q, b);
    if (cbd != acb) return false;
    return orient(r, q, a) == acb;
}

}  // namespace exact
}  // namespace gahhg
