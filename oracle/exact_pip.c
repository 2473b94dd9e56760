/*
 * exact_pip.c - exact point-in-spherical-polygon oracle (TEST INFRASTRUCTURE).
 *
 * Brute force over every polygon edge, exact predicates.  Defines the labels
 * of the library's exact semantics (GAHHG_SEMANTICS_EXACT); the GPU engine is
 * checked against it.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU baseline use it.
 *
 * Definitions (all on the canonical FP64 XYZ of include/gahhg_canon.h):
 *  orient(a,b,c) = sign(det[a;b;c]) = sign(a . (b x c)), evaluated exactly:
 *    an FP64 evaluation with a forward error bound of 8 eps times the
 *    permanent decides when it can; otherwise the determinant is summed
 *    exactly with floating-point expansions (error-free two_sum/two_product,
 *    Shewchuk, "Adaptive Precision Floating-Point Arithmetic and Fast Robust
 *    Geometric Predicates", 1997) and the sign of its largest component is
 *    taken.
 *  Exact zeros are broken by simulation of simplicity (Edelsbrunner & Muecke,
 *    1990): the three points are ranked lexicographically, entry (r, c) of the
 *    ranked matrix is perturbed by eps^(2^(3r+c)), and the sign of the first
 *    non-vanishing coefficient of det(M + E) in increasing order of exponent
 *    is returned.  The rank depends only on coordinates, so the perturbation
 *    is the same in every predicate a point takes part in.  Identical points
 *    cannot be separated; callers never pass them (see below).
 *  Arcs (p,q) and (a,b) cross iff orient(a,r,b) = orient(b,q,a) =
 *    orient(r,b,q) = orient(q,a,r) with r = p (all four equal).
 *  label(q): a point X just left of an outer-ring edge is inside (outer ring
 *    counter-clockwise, holes clockwise, as the loader orients them); six
 *    fixed hub points near +-x, +-y, +-z get their labels by crossing parity
 *    from X; q takes the label of its nearest hub XOR the parity of the polygon
 *    edges crossing arc(hub, q).  Zero-length edges are skipped.  A query
 *    point equal to a polygon vertex is inside.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "gahhg_canon.h"

/* ------------------------------------------------------ expansion arithmetic */

static inline void two_sum(double a, double b, double* s, double* e)
{
    double x = a + b;
    double bv = x - a;
    double av = x - bv;
    *s = x;
    *e = (a - av) + (b - bv);
}

static inline void two_prod(double a, double b, double* p, double* e)
{
    double x = a * b;
    *p = x;
    *e = fma(a, b, -x);
}

/* h = e + b, e of length m (nonoverlapping, increasing magnitude); returns length */
static int grow_expansion(int m, const double* e, double b, double* h)
{
    double q = b;
    int k = 0;
    for (int i = 0; i < m; i++) {
        double s, t;
        two_sum(q, e[i], &s, &t);
        if (t != 0.0) h[k++] = t;
        q = s;
    }
    if (q != 0.0 || k == 0) h[k++] = q;
    return k;
}

static int expansion_sign(int m, const double* e)
{
    for (int i = m - 1; i >= 0; i--) {
        if (e[i] > 0) return 1;
        if (e[i] < 0) return -1;
    }
    return 0;
}

/* exact sign of sum of terms[0..n) (each term exactly representable) */
static int exact_sum_sign(const double* terms, int n)
{
    double a[128], b[128];
    double* cur = a;
    double* nxt = b;
    int m = 0;
    for (int i = 0; i < n; i++) {
        if (terms[i] == 0.0) continue;
        m = grow_expansion(m, cur, terms[i], nxt);
        double* t = cur;
        cur = nxt;
        nxt = t;
    }
    return expansion_sign(m, cur);
}

/* exact a*b*c as 4 terms */
static void triple_prod(double a, double b, double c, double* out)
{
    double p, e;
    two_prod(b, c, &p, &e);
    two_prod(a, p, &out[0], &out[1]);
    two_prod(a, e, &out[2], &out[3]);
}

static int det3_exact_sign(const double* a, const double* b, const double* c)
{
    double t[24];
    /* a0 (b1 c2 - b2 c1) + a1 (b2 c0 - b0 c2) + a2 (b0 c1 - b1 c0) */
    triple_prod(a[0], b[1], c[2], t + 0);
    triple_prod(-a[0], b[2], c[1], t + 4);
    triple_prod(a[1], b[2], c[0], t + 8);
    triple_prod(-a[1], b[0], c[2], t + 12);
    triple_prod(a[2], b[0], c[1], t + 16);
    triple_prod(-a[2], b[1], c[0], t + 20);
    return exact_sum_sign(t, 24);
}

static int det2_exact_sign(double u0, double u1, double v0, double v1)
{
    /* u0 v1 - u1 v0 */
    double t[4];
    two_prod(u0, v1, &t[0], &t[1]);
    two_prod(-u1, v0, &t[2], &t[3]);
    return exact_sum_sign(t, 4);
}

static inline int sgn(double x) { return (x > 0) - (x < 0); }

/* ------------------------------------------------------------ predicates */

#define EPS53 1.1102230246251565e-16 /* 2^-53 */

static int orient_raw(const double* a, const double* b, const double* c)
{
    double m0 = b[1] * c[2] - b[2] * c[1];
    double m1 = b[2] * c[0] - b[0] * c[2];
    double m2 = b[0] * c[1] - b[1] * c[0];
    double d = a[0] * m0 + a[1] * m1 + a[2] * m2;
    double perm = fabs(a[0]) * (fabs(b[1] * c[2]) + fabs(b[2] * c[1])) +
                  fabs(a[1]) * (fabs(b[2] * c[0]) + fabs(b[0] * c[2])) +
                  fabs(a[2]) * (fabs(b[0] * c[1]) + fabs(b[1] * c[0]));
    double bound = 8.0 * EPS53 * perm;
    if (d > bound) return 1;
    if (d < -bound) return -1;
    return det3_exact_sign(a, b, c);
}

static int lex_less(const double* p, const double* q)
{
    if (p[0] != q[0]) return p[0] < q[0];
    if (p[1] != q[1]) return p[1] < q[1];
    return p[2] < q[2];
}

static int same_point(const double* p, const double* q) { return p[0] == q[0] && p[1] == q[1] && p[2] == q[2]; }

/* simulation of simplicity for an exactly vanishing det[a;b;c] */
static int orient_sos(const double* a, const double* b, const double* c)
{
    const double* P[3] = {a, b, c};
    int parity = 0;
    /* sort rows lexicographically, tracking permutation parity */
    for (int i = 0; i < 3; i++)
        for (int j = 0; j + 1 < 3 - i; j++)
            if (lex_less(P[j + 1], P[j])) {
                const double* t = P[j];
                P[j] = P[j + 1];
                P[j + 1] = t;
                parity ^= 1;
            }
    if (same_point(P[0], P[1]) || same_point(P[1], P[2])) return 0;
    static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    static const int psign[6] = {1, -1, -1, 1, 1, -1};
    for (int mask = 1; mask < 512; mask++) {
        int rows = 0, cols = 0, cnt = 0, ok = 1;
        int rc[3][2];
        for (int p = 0; p < 9 && ok; p++) {
            if (!(mask >> p & 1)) continue;
            int r = p / 3, c = p % 3;
            if ((rows >> r & 1) || (cols >> c & 1)) ok = 0;
            rows |= 1 << r;
            cols |= 1 << c;
            rc[cnt][0] = r;
            rc[cnt][1] = c;
            cnt++;
        }
        if (!ok) continue;
        int s = 0;
        if (cnt == 1) {
            int r = rc[0][0], c = rc[0][1];
            int r0 = r == 0 ? 1 : 0, r1 = r == 2 ? 1 : 2;
            int c0 = c == 0 ? 1 : 0, c1 = c == 2 ? 1 : 2;
            s = det2_exact_sign(P[r0][c0], P[r0][c1], P[r1][c0], P[r1][c1]);
            if ((r + c) & 1) s = -s;
        } else {
            /* the permutations containing the chosen entries */
            for (int k = 0; k < 6; k++) {
                int match = 1;
                for (int e = 0; e < cnt; e++)
                    if (perms[k][rc[e][0]] != rc[e][1]) match = 0;
                if (!match) continue;
                if (cnt == 3) {
                    s = psign[k];
                } else {
                    int r3 = 3 - rc[0][0] - rc[1][0];
                    s = psign[k] * sgn(P[r3][perms[k][r3]]);
                }
                break;
            }
        }
        if (s != 0) return parity ? -s : s;
    }
    return 0;
}

int oracle_orient(const double* a, const double* b, const double* c)
{
    int s = orient_raw(a, b, c);
    if (s != 0) return s;
    return orient_sos(a, b, c);
}

int oracle_orient_nosos(const double* a, const double* b, const double* c) { return orient_raw(a, b, c); }

/* arc (r,q) crosses arc (a,b); the four points are pairwise distinct */
int oracle_crossing(const double* r, const double* q, const double* a, const double* b)
{
    int acb = -oracle_orient(a, b, r);
    int bda = oracle_orient(a, b, q);
    if (bda != acb) return 0;
    int cbd = -oracle_orient(r, q, b);
    if (cbd != acb) return 0;
    int dac = oracle_orient(r, q, a);
    return dac == acb;
}

/* -------------------------------------------------------------- polygon */

typedef struct {
    int n;
    const double* pv; /* n x 3, borrowed */
    const int* pe;    /* n x 2, borrowed */
    double x_in[3];
    double hubs[6][3];
    int hub_label[6]; /* 1 = out, 2 = in */
    int ref_edge;
} exact_poly;

static const double HUBS[6][3] = {
    {1.0, 0.000731, 0.000419},  {-1.0, 0.000627, -0.000883}, {0.000577, 1.0, 0.000941},
    {-0.000351, -1.0, 0.000713}, {0.000809, -0.000467, 1.0}, {-0.000689, 0.000523, -1.0},
};

/* parity of edges crossing arc (p, q); -1 if q or p coincides with a vertex */
static int arc_parity(const exact_poly* P, const double* p, const double* q)
{
    int par = 0;
    for (int e = 0; e < P->n; e++) {
        const double* a = P->pv + 3 * P->pe[2 * e];
        const double* b = P->pv + 3 * P->pe[2 * e + 1];
        if (same_point(a, b)) continue;
        if (same_point(q, a) || same_point(q, b) || same_point(p, a) || same_point(p, b)) return -1;
        par ^= oracle_crossing(p, q, a, b);
    }
    return par;
}

static double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* The point just left of an outer edge: exact_reference_point in the GPU engine
 * follows the same steps. */
int oracle_reference_point(const double* pv, const int* pe, int n, int n_outer, double* x_in, int* edge)
{
    exact_poly tmp;
    tmp.n = n;
    tmp.pv = pv;
    tmp.pe = pe;
    for (int e = 0; e < n_outer; e++) {
        const double* a = pv + 3 * pe[2 * e];
        const double* b = pv + 3 * pe[2 * e + 1];
        if (same_point(a, b)) continue;
        double m[3] = {a[0] + b[0], a[1] + b[1], a[2] + b[2]};
        double nm = sqrt(dot3(m, m));
        if (!(nm > 1e-3)) continue; /* near-antipodal endpoints */
        double N[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
        double nn = sqrt(dot3(N, N));
        if (!(nn > 0)) continue;
        double d[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
        double t = 1e-3 * sqrt(dot3(d, d));
        double xi[3], xo[3];
        for (int k = 0; k < 3; k++) {
            xi[k] = m[k] / nm + t * (N[k] / nn);
            xo[k] = m[k] / nm - t * (N[k] / nn);
        }
        if (oracle_orient(a, b, xi) <= 0 || oracle_orient(a, b, xo) >= 0) continue;
        if (arc_parity(&tmp, xo, xi) != 1) continue;
        /* exactly one crossing and it is this edge */
        if (!oracle_crossing(xo, xi, a, b)) continue;
        memcpy(x_in, xi, sizeof(xi));
        *edge = e;
        return 0;
    }
    return -1;
}

static int nearest_hub(const double* q)
{
    int best = 0;
    double bd = -1e300;
    for (int k = 0; k < 6; k++) {
        double d = dot3(HUBS[k], q);
        if (d > bd) {
            bd = d;
            best = k;
        }
    }
    return best;
}

void* exact_poly_new(const double* pv, const int* pe, int n, int n_outer)
{
    exact_poly* P = (exact_poly*)calloc(1, sizeof(exact_poly));
    P->n = n;
    P->pv = pv;
    P->pe = pe;
    memcpy(P->hubs, HUBS, sizeof(HUBS));
    if (oracle_reference_point(pv, pe, n, n_outer, P->x_in, &P->ref_edge) != 0) {
        free(P);
        return NULL;
    }
    for (int k = 0; k < 6; k++) P->hub_label[k] = 0;
    int h0 = nearest_hub(P->x_in);
    int par = arc_parity(P, P->x_in, HUBS[h0]);
    if (par < 0) {
        free(P);
        return NULL;
    }
    P->hub_label[h0] = par ? 1 : 2;
    int opp = h0 ^ 1;
    for (int k = 0; k < 6; k++) {
        if (k == h0 || k == opp) continue;
        int pk = arc_parity(P, HUBS[h0], HUBS[k]);
        if (pk < 0) {
            free(P);
            return NULL;
        }
        P->hub_label[k] = pk ? 3 - P->hub_label[h0] : P->hub_label[h0];
    }
    int via = (h0 + 2) % 6;
    int po = arc_parity(P, HUBS[via], HUBS[opp]);
    if (po < 0) {
        free(P);
        return NULL;
    }
    P->hub_label[opp] = po ? 3 - P->hub_label[via] : P->hub_label[via];
    return P;
}

void exact_poly_free(void* h) { free(h); }

void exact_poly_info(const void* h, double* x_in, double* hubs, int* hub_labels, int* ref_edge)
{
    const exact_poly* P = (const exact_poly*)h;
    if (x_in) memcpy(x_in, P->x_in, sizeof(P->x_in));
    if (hubs) memcpy(hubs, P->hubs, sizeof(P->hubs));
    if (hub_labels) memcpy(hub_labels, P->hub_label, sizeof(P->hub_label));
    if (ref_edge) *ref_edge = P->ref_edge;
}

static uint8_t label_xyz(const exact_poly* P, const double* q)
{
    for (int e = 0; e < P->n; e++) {
        const double* a = P->pv + 3 * P->pe[2 * e];
        if (same_point(q, a)) return 2;
    }
    int h = nearest_hub(q);
    if (same_point(q, HUBS[h])) return (uint8_t)P->hub_label[h];
    int par = arc_parity(P, HUBS[h], q);
    int l = P->hub_label[h];
    return (uint8_t)(par ? 3 - l : l);
}

void exact_poly_query_xyz(const void* h, const double* q, long n, uint8_t* out, int threads)
{
    const exact_poly* P = (const exact_poly*)h;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads > 0 ? threads : 1)
    for (long i = 0; i < n; i++) out[i] = label_xyz(P, q + 3 * i);
}

void exact_poly_query_lonlat(const void* h, const double* lonlat, long n, uint8_t* out, int threads)
{
    const exact_poly* P = (const exact_poly*)h;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads > 0 ? threads : 1)
    for (long i = 0; i < n; i++) {
        double q[3];
        gahhg_canon_query_xyz(lonlat[2 * i], lonlat[2 * i + 1], q);
        out[i] = label_xyz(P, q);
    }
}

/* parity of polygon edges crossing arc (p, q); -1 on vertex coincidence */
int exact_poly_arc_parity(const void* h, const double* p, const double* q)
{
    return arc_parity((const exact_poly*)h, p, q);
}

void oracle_canon_query_xyz(const double* lonlat, long n, double* xyz)
{
    for (long i = 0; i < n; i++) gahhg_canon_query_xyz(lonlat[2 * i], lonlat[2 * i + 1], xyz + 3 * i);
}

void oracle_canon_vertex_xyz(const double* lonlat, long n, double* xyz)
{
    for (long i = 0; i < n; i++) gahhg_canon_vertex_xyz(lonlat[2 * i], lonlat[2 * i + 1], xyz + 3 * i);
}

/* side[6 e + k] = orient(a_e, b_e, hub_k) for every edge (the exact signs
 * the GPU brute force, oracle/brute_gpu.cu, takes as given). */
void exact_poly_hub_sides(const void* h, signed char* side, int threads)
{
    const exact_poly* P = (const exact_poly*)h;
#pragma omp parallel for schedule(static) num_threads(threads > 0 ? threads : 1)
    for (int e = 0; e < P->n; e++) {
        const double* a = P->pv + 3 * P->pe[2 * e];
        const double* b = P->pv + 3 * P->pe[2 * e + 1];
        for (int k = 0; k < 6; k++) side[6 * (long)e + k] = (signed char)oracle_orient(a, b, P->hubs[k]);
    }
}
