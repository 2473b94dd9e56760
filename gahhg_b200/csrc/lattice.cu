// lattice.cu - exact-label query index and query kernel.
//
// The reference answers a query by descending the hexagon hierarchy from 42
// level-0 cells (kernel_PISP, source/GPISPAHHG.cu:1422-1504): about ten
// dependent levels of plane tests per point.  Here the same question is
// answered from a lattice over longitude/latitude that is indexed directly
// from the input coordinates:
//
//   * top level: W x H cells of equal angular size (H = W/2) covering
//     lon [-180,180) x lat [-90,90]; a cell's region is its rectangle of
//     (lon, lat) mapped through the canonical conversion;
//   * each cell owns a cap (center R = canonical XYZ of the cell center,
//     radius 2 * (half-height + half-width * cos(center lat)) + margin), which
//     contains the cell, every point within the margin of it, and the caps of
//     all its descendants; a polygon edge is listed in a cell when it may meet
//     the cap (conservative test);
//   * a cell listing more than K edges is split 4 x 4, down to a depth limit;
//   * every cell center has an exact label: the top row and each column are
//     chained by the crossing parity of the arc between neighbouring centers
//     (both ends lie in the union of the two caps), the first center is
//     reached from a point just left of an outer-ring edge through six fixed
//     hub points, and a child takes its parent's label XOR the parity of the
//     arc parent-center -> child-center against the parent's edges.
//
// A query reads lon/lat (16 B), computes the top cell with two FP64
// multiply-adds, follows inner nodes by exact power-of-two scaling, and
//   - in a cell without edges writes the cell's label (no trigonometry);
//   - in a leaf counts crossings of arc(R, q) with the leaf's edges:
//       s2 = orient(A,B,q) = q.(A x B), s3 = orient(R,q,A) = q.(A x R),
//       s4 = orient(R,q,B) = q.(B x R), s1 = orient(A,B,R) stored exactly;
//     each sign is first taken in FP32 (q from __sincosf, vectors rounded to
//     FP32) against a forward error bound, then in FP64 on the canonical q,
//     then exactly (exact_pred.cuh).  Labels are therefore those of the exact
//     oracle; the FP32 stage only decides when its bound proves the sign.
#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <thread>
#include <type_traits>
#include <vector>

#include "exact_pred.cuh"
#include "gahhg_canon.h"
#include "gahhg_internal.h"
#include "local_frame.cuh"

namespace gahhg {

namespace {

constexpr int TPB = 256;
inline int blocks_for(long long n) { return (int)std::max(1LL, (n + TPB - 1) / TPB); }

constexpr int FAN = 4;                     // children per axis
constexpr uint32_t KIND_MASK = 0xC0000000u;
constexpr uint32_t KIND_PURE = 0x00000000u;  // low bits: label (1 out, 2 in)
constexpr uint32_t KIND_INNER = 0x80000000u;  // low 30 bits: first child node
constexpr uint32_t KIND_LEAF = 0xC0000000u;  // low 30 bits: leaf index
constexpr uint32_t INDEX_MASK = 0x3FFFFFFFu;

// Margin (radians) between where the index arithmetic places a query and
// where its canonical XYZ lies: index rounding (~1e-14), conversion error
// (~1e-15), longitudes up to +-540 (2 pi' differs from 2 pi by 7.2e-9).
constexpr double LOC_MARGIN = 2.0e-8;
constexpr double RAD = GAHHG_PI_TRUNC / 180.0;  // degrees -> canonical radians (approx., bounds only)

// Cap radius = CAP_FACTOR x (half-height + half-width x cos(center lat)).
// hlat + hlon cos(lat) bounds the distance from the center to any point of
// the cell (along a parallel, then a meridian).  Children of a 4 x 4 split
// have their centers within 3/4 of that bound from the parent's center and
// bounds of about a quarter of it, so a factor of 1.25 keeps every child cap
// inside its parent's cap with room for the distortion near the poles (the
// build checks every child), and the arc between two neighbouring top-level
// centers stays inside the union of their caps.
constexpr double CAP_FACTOR = 1.25;

// Refinement limits: node words (4 B each) and edge entries of one level.
constexpr long long NODE_BUDGET = 1LL << 27;
constexpr long long PAIR_BUDGET = 1LL << 30;

// Leaf: its center as the lon/lat it was placed at (R = their canonical XYZ,
// recomputed where needed), its edge records, its center's label, and the
// sine and cosine of the center's canonical latitude rounded to float (the
// FP32 tier's frame, local_frame::frame_at).  32 bytes: one sector.
struct __align__(16) LeafRec {
    double lon, lat;
    uint32_t off;
    uint16_t cnt;
    uint8_t label;
    uint8_t pad;
    float sb, cb;
};
static_assert(sizeof(LeafRec) == 32, "LeafRec");

// (leaf, edge) records of the FP32 tier: float4 (a1, a2, b1, b2), the edge's
// ends in the leaf's tangent frame (local_frame::edge_record), ordered so that
// orient(A, B, R) = +1.  The edge id and the sign of orient(A, B, R) in the
// edge's own order are in a parallel array of words (edge | (sign > 0) << 31).

// Level-0 grid over a lon/lat domain: W x H cells of dlon0 x dlat0 degrees
// starting at (lon0, lat0).  full_lon: the domain spans all longitudes
// (W * dlon0 = 360); to_north / to_south: it reaches the pole.  cap_cos
// bounds cos(latitude) over the domain (1 when it spans the equator).
struct Geo {
    int W, H;
    double lon0, lat0;
    double dlon0, dlat0;
    double cap_cos;
    bool full_lon, to_north, to_south;
};

// A polygon of a group build: its level-0 grid, first top node, leaf size
// and first edge in the group's arrays.
struct PolyGeo {
    Geo g;
    long long top;
    int K;
    int e0;
};

// The level-0 grid of a node's polygon: the build's one polygon, or a group
// build's polygon table through the level's node -> polygon array; top() is
// the polygon's first top node (child indices in node words are relative to
// it).
struct OneGeo {
    Geo g;
    __device__ __forceinline__ const Geo& of(long long) const { return g; }
    __device__ __forceinline__ long long top(long long) const { return 0; }
};
struct TableGeo {
    const PolyGeo* pg;
    const int* npoly;
    __device__ __forceinline__ const Geo& of(long long v) const { return pg[npoly[v]].g; }
    __device__ __forceinline__ long long top(long long v) const { return pg[npoly[v]].top; }
};

// Node geometry from (level, ix, iy): center (degrees, exact), cap radius.
struct NodeCap {
    double R[3];
    double r;
    double lonc, latc;
};

__host__ __device__ inline double level_scale(int lvl)
{
    double s = 1.0;
    for (int i = 0; i < lvl; i++) s *= FAN;
    return s;
}

__host__ __device__ inline NodeCap node_cap(const Geo& g, int lvl, long long ix, long long iy)
{
    const double sc = level_scale(lvl);
    const double dlon = g.dlon0 / sc, dlat = g.dlat0 / sc;
    NodeCap c;
    c.lonc = g.lon0 + ((double)ix + 0.5) * dlon;
    c.latc = g.lat0 + ((double)iy + 0.5) * dlat;
    gahhg_canon_vertex_xyz(c.lonc, c.latc, c.R);
    // the width term takes cos at the cell's equator-ward edge, the widest
    // parallel of the cell: a child's center then lies within 3/4 of the
    // parent's bound and its own bound is a quarter of it, so every child cap
    // nests in its parent's for any cell aspect (near a pole cos changes by a
    // large factor across one cell)
    const double phi_eq = fmax(fabs(c.latc) - 0.5 * dlat, 0.0);
    double sa, ca;
    gahhg_canon_sincos(gahhg_canon_rad(phi_eq), &sa, &ca);
    const double hlat = 0.5 * dlat * RAD, hlon = 0.5 * dlon * RAD;
    c.r = CAP_FACTOR * (hlat + hlon * fabs(ca)) * (1.0 + 1e-9) + LOC_MARGIN + 1e-12;
    return c;
}

// Moves R off a polygon vertex it coincides with (exact comparison).
__host__ __device__ inline void nudge_center(const Geo& g, int lvl, NodeCap& c, const D3* pv, const int* pe,
                                             const int* list, int cnt)
{
    const double sc = level_scale(lvl);
    for (int tries = 0; tries < 8; tries++) {
        bool hit = false;
        for (int k = 0; k < cnt && !hit; k++) {
            const int e = list[k];
            const D3 a = pv[pe[2 * e]], b = pv[pe[2 * e + 1]];
            hit = (a.x == c.R[0] && a.y == c.R[1] && a.z == c.R[2]) || (b.x == c.R[0] && b.y == c.R[1] && b.z == c.R[2]);
        }
        if (!hit) return;
        c.lonc += g.dlon0 / sc * (1.0 / 1024.0);
        c.latc += g.dlat0 / sc * (1.0 / 2048.0);
        gahhg_canon_vertex_xyz(c.lonc, c.latc, c.R);
    }
}

// The cap's thresholds: squared chord of its radius r and the bound on the
// sine of the distance from its center to a great circle that meets it.
__host__ __device__ inline double cap_chord2(double r)
{
    const double chord = 2.0 * sin(0.5 * r) * (1.0 + 1e-9) + 1e-12;
    return chord * chord;
}
__host__ __device__ inline double cap_sin_bound(double r) { return sin(r) * (1.0 + 1e-9) + 1e-12; }

// edge_hits_cap with the cap's thresholds and the edge's normal N = A x B,
// nn = |N|, computed once by the caller.
__host__ __device__ inline bool edge_hits_cap_pre(const D3& A, const D3& B, const D3& N, double nn, const double* R,
                                                  double c2, double sb)
{
    const double ax = A.x - R[0], ay = A.y - R[1], az = A.z - R[2];
    if (ax * ax + ay * ay + az * az <= c2) return true;
    const double bx = B.x - R[0], by = B.y - R[1], bz = B.z - R[2];
    if (bx * bx + by * by + bz * bz <= c2) return true;
    if (!(nn > 1e-300)) return false;
    const double s = (N.x * R[0] + N.y * R[1] + N.z * R[2]) / nn;
    if (fabs(s) > sb) return false;
    const D3 Rv = d3(R[0], R[1], R[2]);
    const double t1 = dot(cross(N, A), Rv), t2 = dot(cross(B, N), Rv);
    const double tol = 1e-12 * nn;
    return t1 >= -tol && t2 >= -tol;
}

// Conservative: may arc AB (unit vectors) come within angle r of R?
__host__ __device__ inline bool edge_hits_cap(const D3& A, const D3& B, const double* R, double r)
{
    const D3 N = cross(A, B);
    return edge_hits_cap_pre(A, B, N, sqrt(dot(N, N)), R, cap_chord2(r), cap_sin_bound(r));
}

__host__ __device__ inline double lat_of(const D3& p) { return asin(fmin(1.0, fmax(-1.0, p.y))) / RAD; }
__host__ __device__ inline double lon_of(const D3& p) { return atan2(p.x, p.z) / RAD; }

// Latitude/longitude box (degrees) of arc AB; full_lon when it may cross a pole.
__host__ __device__ inline void arc_box(const D3& A, const D3& B, double& la0, double& la1, double& lo0, double& lo1,
                               bool& full_lon)
{
    double a = lat_of(A), b = lat_of(B);
    la0 = fmin(a, b);
    la1 = fmax(a, b);
    const D3 N = cross(A, B);
    const double nn = sqrt(dot(N, N));
    if (nn > 1e-300) {
        const D3 n = N * (1.0 / nn);
        D3 V = d3(-n.y * n.x, 1.0 - n.y * n.y, -n.y * n.z);  // highest point of the great circle
        const double vv = sqrt(dot(V, V));
        if (vv > 1e-300) {
            V = V * (1.0 / vv);
            for (int sgn = 0; sgn < 2; sgn++) {
                const D3 P = sgn ? -V : V;
                if (dot(cross(N, A), P) >= 0 && dot(cross(B, N), P) >= 0) {
                    const double lp = lat_of(P);
                    la0 = fmin(la0, lp);
                    la1 = fmax(la1, lp);
                }
            }
        }
    }
    full_lon = false;
    double oa = lon_of(A), ob = lon_of(B);
    if (fabs(a) > 89.999 || fabs(b) > 89.999 || la1 > 89.99 || la0 < -89.99) {
        full_lon = true;
        lo0 = -180;
        lo1 = 180;
        return;
    }
    if (oa > ob) {
        double t = oa;
        oa = ob;
        ob = t;
    }
    if (ob - oa <= 180.0) {
        lo0 = oa;
        lo1 = ob;
    } else {
        lo0 = ob;
        lo1 = oa + 360.0;
    }
}

struct BuildView {
    Geo g;
    const D3* pv;
    const int* pe;
    int n;
};

// Level-0 candidates of one edge: rows [iy0, iy0 + nrows) by up to two
// column ranges [c0, c0 + n0) and [c1, c1 + n1) (the inflated longitude
// interval may wrap past 360 degrees relative to the domain's west edge).
struct EdgeBox {
    int iy0, nrows, c0, n0, c1, n1;
};

// A work item is one row of one column chunk of an edge's box, so no thread
// tests more than L0_CHUNK cells: an edge near a pole (all columns) or a
// very long edge has a box of up to millions of cells, and one thread per
// edge would hold its block for tens of milliseconds.
constexpr int L0_CHUNK = 64;
// Work items whose hit masks the count pass keeps for the fill pass (8 bytes
// each; beyond this the fill pass tests again).
constexpr unsigned long long L0_MASK_ITEMS = 1ull << 26;

__device__ inline int l0_chunks(int n) { return (n + L0_CHUNK - 1) / L0_CHUNK; }

// Per edge: its candidate box and number of work items; total64 accumulates
// the 64-bit item total (the 32-bit scan of the counts must not wrap).
// Candidate box of edge AB in the level-0 grid g; returns its work items.
__device__ long long edge_box(const Geo& g, const D3& A, const D3& B, EdgeBox& bx)
{
    const int W = g.W, H = g.H;
    double la0, la1, lo0, lo1;
    bool full;
    arc_box(A, B, la0, la1, lo0, lo1, full);
    const double rmax = (CAP_FACTOR * (0.5 * g.dlat0 + 0.5 * g.dlon0 * g.cap_cos) * RAD) * (1.0 + 1e-6) + LOC_MARGIN;
    const double rdeg = rmax / RAD + 1e-9;
    la0 -= rdeg;
    la1 += rdeg;
    int iy0 = (int)floor((la0 - g.lat0) / g.dlat0), iy1 = (int)floor((la1 - g.lat0) / g.dlat0);
    iy0 = max(iy0, 0);
    iy1 = min(iy1, H - 1);
    const double maxlat = fmax(fabs(la0), fabs(la1));
    long long r0a = 0, r0b = W - 1, r1a = 1, r1b = 0;
    bool all_cols = full || maxlat >= 89.0;
    if (!all_cols) {
        const double c = cos(maxlat * RAD);
        const double wdeg = rdeg / c;
        const double len = (lo1 - lo0) + 2 * wdeg;
        if (len >= 360.0) {
            all_cols = true;
        } else {
            double a = lo0 - wdeg - g.lon0;
            a -= 360.0 * floor(a / 360.0);  // [0, 360)
            r0a = (long long)floor(a / g.dlon0);
            r0b = (long long)floor((a + len) / g.dlon0);
            if (a + len >= 360.0) {
                r1a = 0;
                r1b = (long long)floor((a + len - 360.0) / g.dlon0);
            }
        }
    }
    if (all_cols) {
        r0a = 0;
        r0b = W - 1;
        r1a = 1;
        r1b = 0;
    }
    r0a = max(r0a, 0LL);
    r0b = min(r0b, (long long)W - 1);
    r1b = min(r1b, (long long)W - 1);
    bx.iy0 = iy0;
    bx.nrows = max(0, iy1 - iy0 + 1);
    bx.c0 = (int)r0a;
    bx.n0 = (int)max(0LL, r0b - r0a + 1);
    bx.c1 = (int)r1a;
    bx.n1 = (int)max(0LL, r1b - r1a + 1);
    return (long long)bx.nrows * (l0_chunks(bx.n0) + l0_chunks(bx.n1));
}

__global__ void k_l0_box(BuildView v, EdgeBox* box, int* items, unsigned long long* total64)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    long long nit = 0;
    if (t < v.n) {
        EdgeBox bx{0, 0, 0, 0, 0, 0};
        const D3 A = v.pv[v.pe[2 * t]], B = v.pv[v.pe[2 * t + 1]];
        if (!(A.x == B.x && A.y == B.y && A.z == B.z)) nit = edge_box(v.g, A, B, bx);
        box[t] = bx;
        items[t] = (int)min(nit, (long long)INT_MAX);
    }
    // one 64-bit atomic per warp
    unsigned long long w = (unsigned long long)nit;
    for (int o = 16; o > 0; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd(total64, w);
}

// Level-0 pairs over the work items (persistent grid; the item total is read
// on the device).  PASS 0 counts per cell, PASS 1 fills the lists.
// The level-0 grid of an edge's polygon (the build's one, or a group's
// table through the edge -> polygon array).
struct EdgeGeoTable {
    const PolyGeo* pg;
    const int* epoly;
    __device__ __forceinline__ const Geo& of(long long e) const { return pg[epoly[e]].g; }
    __device__ __forceinline__ long long top(long long e) const { return pg[epoly[e]].top; }
};

// Level-0 pairs over the work items (persistent grid; the item total is read
// on the device).  PASS 0 tests an item's cells (at most L0_CHUNK) and counts
// per cell, recording the item's hits in mask[it] when mask is given; PASS 1
// fills the lists from those masks (or tests again without them).
template <int PASS, class GEO>
__global__ void k_l0_expand(const D3* __restrict__ pv, const int* __restrict__ pe, long long ne, GEO geo,
                            const EdgeBox* __restrict__ box, const int* __restrict__ item_off,
                            const int* total_items, const unsigned long long* total64, int* cnt, const int* off,
                            int* cursor, int* list, unsigned long long* mask)
{
    static_assert(L0_CHUNK <= 64, "a 64-bit hit mask per item");
    if (*total64 > (unsigned long long)INT_MAX) return;  // the host reports it; the 32-bit offsets wrapped
    const int total = *total_items;
    for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < total; it += gridDim.x * blockDim.x) {
        unsigned long long m = 0;
        if (PASS == 1 && mask) {
            m = mask[it];
            if (!m) continue;
        }
        long long lo = 0, hi = ne;  // the last edge whose first item is <= it
        while (hi - lo > 1) {
            const long long mid = (lo + hi) >> 1;
            if (item_off[mid] <= it) lo = mid;
            else hi = mid;
        }
        const long long t = lo;
        const EdgeBox b = box[t];
        const Geo& G = geo.of(t);
        const int W = G.W, H = G.H;
        const int k0 = l0_chunks(b.n0), kk = k0 + l0_chunks(b.n1);
        const int local = it - item_off[t];
        const int iy = kk ? b.iy0 + local / kk : -1;
        const int ch = kk ? local % kk : 0;
        int xa, xb;
        if (ch < k0) {
            xa = b.c0 + ch * L0_CHUNK;
            xb = min(b.c0 + b.n0, xa + L0_CHUNK);
        } else {
            xa = b.c1 + (ch - k0) * L0_CHUNK;
            xb = min(b.c1 + b.n1, xa + L0_CHUNK);
        }
        if (iy < 0 || iy >= H || xa < 0 || xb > W) {
            if (PASS == 0 && mask) mask[it] = 0;
            continue;
        }
        const long long row = geo.top(t) + (long long)iy * W;
        if (PASS == 0 || !mask) {
            const D3 A = pv[pe[2 * t]], B = pv[pe[2 * t + 1]];
            for (int ix = xa; ix < xb; ix++) {
                const NodeCap c = node_cap(G, 0, ix, iy);
                if (edge_hits_cap(A, B, c.R, c.r)) m |= 1ull << (ix - xa);
            }
        }
        if (PASS == 0) {
            if (mask) mask[it] = m;
            for (unsigned long long r = m; r; r &= r - 1) atomicAdd(&cnt[row + xa + __ffsll((long long)r) - 1], 1);
        } else {
            for (unsigned long long r = m; r; r &= r - 1) {
                const long long node = row + xa + __ffsll((long long)r) - 1;
                list[off[node] + atomicAdd(&cursor[node], 1)] = (int)t;
            }
        }
    }
}

// Cap of every child node of a level, once: center R and the squared chord
// in caps, the sine bound and the radius in capsb (cap_chord2 /
// cap_sin_bound of its radius).
__global__ void k_child_caps(Geo g, int lvl, int nn, const long long* ix, const long long* iy, double4* caps,
                             double2* capsb)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nn) return;
    const NodeCap nc = node_cap(g, lvl, ix[c], iy[c]);
    caps[c] = make_double4(nc.R[0], nc.R[1], nc.R[2], cap_chord2(nc.r));
    capsb[c] = make_double2(cap_sin_bound(nc.r), nc.r);
}

// Children pairs, count pass: one thread per (refined parent, edge) pair
// tests the parent's FAN x FAN children (consecutive nodes) and records its
// hits as a mask, so the fill pass writes the list entries without testing
// again.  (Sixteen lanes per pair, one child each, ran 2.2x slower on the C1
// polygon: a pair is only sixteen tests, and the dependent loads that start
// it were then paid by a half-warp instead of one thread.)
__global__ void __launch_bounds__(TPB) k_child_pairs_count(BuildView v, int npairs, const int* __restrict__ pair_node,
                                                           const int* __restrict__ plist,
                                                           const int* __restrict__ child_base,
                                                           const double4* __restrict__ caps,
                                                           const double2* __restrict__ capsb, int cstart, int* cnt,
                                                           uint16_t* hit)
{
    static_assert(FAN * FAN == 16, "a 16-bit hit mask per pair");
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= npairs) return;
    const int cb = child_base[pair_node[k]];
    if (cb < 0) return;
    const int e = plist[k];
    const D3 A = v.pv[v.pe[2 * e]], B = v.pv[v.pe[2 * e + 1]];
    const D3 N = cross(A, B);
    const double nn = sqrt(dot(N, N));
    unsigned int m = 0;
    for (int l = 0; l < FAN * FAN; l++) {
        const int node = cb + l - cstart;
        const double4 c = caps[node];
        const double R[3] = {c.x, c.y, c.z};
        if (!edge_hits_cap_pre(A, B, N, nn, R, c.w, capsb[node].x)) continue;
        m |= 1u << l;
        atomicAdd(&cnt[node], 1);
    }
    hit[k] = (uint16_t)m;
}

// Children pairs, fill pass: one thread per pair, one entry per hit.
__global__ void k_child_pairs_fill(int npairs, const int* __restrict__ pair_node, const int* __restrict__ plist,
                                   const int* __restrict__ child_base, int cstart, const uint16_t* __restrict__ hit,
                                   const int* off, int* cursor, int* list)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= npairs) return;
    const int cb = child_base[pair_node[k]];
    if (cb < 0) return;
    unsigned int m = hit[k];
    const int e = plist[k];
    while (m) {
        const int l = __ffs(m) - 1;
        m &= m - 1u;
        const int node = cb + l - cstart;
        list[off[node] + atomicAdd(&cursor[node], 1)] = e;
    }
}

__global__ void k_fill_pair_node(const int* cnt, const int* off, int nn, int* pair_node)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nn) return;
    for (int k = 0; k < cnt[p]; k++) pair_node[off[p] + k] = p;
}

// Cell lists are filled with atomics, so their order is arbitrary; sorting
// makes the index deterministic.  Short lists are sorted by their own thread;
// longer ones are handed to k_sort_long, where a whole block sorts each, so
// no thread spends O(n^2) steps on one list.
constexpr int SORT_SMALL = 64;
constexpr int SORT_SMEM = 12256;  // ints staged in shared memory (48 KB with the block's counter)
constexpr int SORT_TPB = 512;

__global__ void k_sort_lists(const int* cnt, const int* off, int nn, int* list, int* long_ids, int* nlong)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nn) return;
    const int n = cnt[p];
    if (n > SORT_SMALL) {
        long_ids[atomicAdd(nlong, 1)] = p;
        return;
    }
    int* L = list + off[p];
    for (int i = 1; i < n; i++) {
        int x = L[i], j = i - 1;
        while (j >= 0 && L[j] > x) {
            L[j + 1] = L[j];
            j--;
        }
        L[j + 1] = x;
    }
}

// Block-wide bitonic sort, ascending, of a[0..n) in the form where every
// comparator puts the minimum at the lower index (the first step of each
// merge compares mirrored positions).  Positions >= n act as +infinity, so
// comparators that reach them are skipped and no padding is stored.
__device__ void block_bitonic_sort(int* a, int n)
{
    int lg = 1;
    while ((1 << lg) < n) lg++;
    const int half = 1 << (lg - 1);  // comparators per step
    for (int lk = 1; lk <= lg; lk++) {
        const int k = 1 << lk;
        for (int lj = lk - 1; lj >= 0; lj--) {
            const int j = 1 << lj;
            for (int t = threadIdx.x; t < half; t += blockDim.x) {
                int i, q;
                if (lj == lk - 1) {  // mirrored compare across the two sorted halves
                    const int base = (t >> lj) << lk, pp = t & (j - 1);
                    i = base + pp;
                    q = base + k - 1 - pp;
                } else {
                    i = ((t >> lj) << (lj + 1)) + (t & (j - 1));
                    q = i + j;
                }
                if (q < n) {
                    const int x = a[i], y = a[q];
                    if (x > y) {
                        a[i] = y;
                        a[q] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// One list per block iteration (a persistent grid takes them from a counter):
// in shared memory up to SORT_SMEM entries, in place in global memory beyond.
__global__ void __launch_bounds__(SORT_TPB) k_sort_long(const int* cnt, const int* off, int* list,
                                                        const int* long_ids, const int* nlong, int* next)
{
    __shared__ int sm[SORT_SMEM];
    __shared__ int s_i;
    const int m = *nlong;
    for (;;) {
        if (threadIdx.x == 0) s_i = atomicAdd(next, 1);
        __syncthreads();
        const int i = s_i;
        if (i >= m) break;
        const int p = long_ids[i];
        const int n = cnt[p];
        int* L = list + off[p];
        if (n <= SORT_SMEM) {
            for (int k = threadIdx.x; k < n; k += blockDim.x) sm[k] = L[k];
            __syncthreads();
            block_bitonic_sort(sm, n);
            for (int k = threadIdx.x; k < n; k += blockDim.x) L[k] = sm[k];
        } else {
            block_bitonic_sort(L, n);
        }
        __syncthreads();
    }
}

__global__ void k_refine_flags(const int* cnt, int nn, int K, int* flag)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < nn) flag[p] = cnt[p] > K ? 1 : 0;
}

// child_base[p] = first child node (global index) or -1; child coordinates.
__global__ void k_make_children(const int* flag, const int* foff, int nn, int cstart, const long long* pix,
                                const long long* piy, int lvl0_W, int* child_base, long long* cix, long long* ciy)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nn) return;
    if (!flag[p]) {
        child_base[p] = -1;
        return;
    }
    const int base = cstart + foff[p] * FAN * FAN;
    child_base[p] = base;
    const long long px = pix ? pix[p] : (p % lvl0_W), py = piy ? piy[p] : (p / lvl0_W);
    for (int cy = 0; cy < FAN; cy++)
        for (int cx = 0; cx < FAN; cx++) {
            const int c = foff[p] * FAN * FAN + cy * FAN + cx;
            cix[c] = px * FAN + cx;
            ciy[c] = py * FAN + cy;
        }
}

__global__ void k_l0_coords(int W, int nn, long long* ix, long long* iy)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nn) return;
    ix[p] = p % W;
    iy[p] = p / W;
}

// parity of edges (from up to two sorted lists, union) crossing arc P->Q
__device__ int arc_parity_lists(const D3* pv, const int* pe, const double* P, const double* Q, const int* L1, int n1,
                                const int* L2, int n2, int* bad)
{
    int par = 0, i = 0, j = 0;
    while (i < n1 || j < n2) {
        int e;
        if (j >= n2 || (i < n1 && L1[i] < L2[j])) {
            e = L1[i++];
        } else if (i >= n1 || L2[j] < L1[i]) {
            e = L2[j++];
        } else {
            e = L1[i];
            i++;
            j++;
        }
        const D3 a = pv[pe[2 * e]], b = pv[pe[2 * e + 1]];
        const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z};
        if (exact::same(A, B)) continue;
        if (exact::same(A, P) || exact::same(B, P) || exact::same(A, Q) || exact::same(B, Q)) {
            atomicAdd(bad, 1);
            continue;
        }
        par ^= exact::crossing(P, Q, A, B) ? 1 : 0;
    }
    return par;
}

// Level-0 neighbour parities: vertical (i,j)->(i,j+1) for all, horizontal on row 0.
__global__ void k_l0_neighbour_parity(BuildView v, const int* cnt, const int* off, const int* list, uint8_t* vpar,
                                      uint8_t* hpar, int* bad)
{
    const int W = v.g.W, H = v.g.H;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nv = (long long)W * (H - 1);
    if (t < nv) {
        const int i = (int)(t % W), j = (int)(t / W);
        const int p = j * W + i, q = (j + 1) * W + i;
        uint8_t par = 0;
        if (cnt[p] || cnt[q]) {
            NodeCap a = node_cap(v.g, 0, i, j), b = node_cap(v.g, 0, i, j + 1);
            nudge_center(v.g, 0, a, v.pv, v.pe, list + off[p], cnt[p]);
            nudge_center(v.g, 0, b, v.pv, v.pe, list + off[q], cnt[q]);
            par = (uint8_t)arc_parity_lists(v.pv, v.pe, a.R, b.R, list + off[p], cnt[p], list + off[q], cnt[q], bad);
        }
        vpar[t] = par;
    } else if (t < nv + W - 1) {
        const int i = (int)(t - nv);
        const int p = i, q = i + 1;
        uint8_t par = 0;
        if (cnt[p] || cnt[q]) {
            NodeCap a = node_cap(v.g, 0, i, 0), b = node_cap(v.g, 0, i + 1, 0);
            nudge_center(v.g, 0, a, v.pv, v.pe, list + off[p], cnt[p]);
            nudge_center(v.g, 0, b, v.pv, v.pe, list + off[q], cnt[q]);
            par = (uint8_t)arc_parity_lists(v.pv, v.pe, a.R, b.R, list + off[p], cnt[p], list + off[q], cnt[q], bad);
        }
        hpar[i] = par;
    }
}

// labels of level-0 centers: row 0 by prefix XOR of hpar, columns by vpar
__global__ void k_l0_labels(int W, int H, const uint8_t* vpar, const uint8_t* hpar, const int* origin_label,
                            uint8_t* label)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= W) return;
    int l = *origin_label;  // 1 or 2
    for (int k = 0; k < i; k++)
        if (hpar[k]) l = 3 - l;
    label[i] = (uint8_t)l;
    for (int j = 1; j < H; j++) {
        if (vpar[(long long)(j - 1) * W + i]) l = 3 - l;
        label[(long long)j * W + i] = (uint8_t)l;
    }
}

// child label = parent label XOR parity(arc parent center -> child center)
// true when R coincides with an end of an edge of the list (nudge_center
// would move it)
__device__ __forceinline__ bool center_on_vertex(const double* R, const D3* pv, const int* pe, const int* list,
                                                 int cnt)
{
    for (int k = 0; k < cnt; k++) {
        const int e = list[k];
        const D3 a = pv[pe[2 * e]], b = pv[pe[2 * e + 1]];
        if ((a.x == R[0] && a.y == R[1] && a.z == R[2]) || (b.x == R[0] && b.y == R[1] && b.z == R[2])) return true;
    }
    return false;
}

// Child labels: parent label XOR the crossing parity of arc(parent center P,
// child center Q) against the parent's list (exact predicates), as
// arc_parity_lists computes it.  A parent's FAN x FAN children are
// consecutive and nchild is a multiple of 16, so each 16-lane group of a
// warp holds one parent's children: its first lane places the parent's
// center and shares it, and the lanes share the children-independent half of
// every crossing test, orient(A, B, P), computed by lane k mod 16 for edge
// k.  Child centers come from the pair pass's caps (node_cap, recomputed
// only when a center must be nudged off a vertex).
template <class GEO>
__global__ void __launch_bounds__(TPB) k_child_labels(BuildView v, GEO geo, int lvl, int nchild, const int* child_parent,
                                                      const long long* cix, const long long* ciy, const int* ccnt,
                                                      const int* coff, const int* clist,
                                                      const double4* __restrict__ ccaps,
                                                      const double2* __restrict__ ccapsb, const long long* pix,
                                                      const long long* piy, const int* pcnt, const int* poff,
                                                      const int* plist, const uint8_t* plabel, uint8_t* clabel,
                                                      int* bad)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nchild) return;
    const int p = child_parent[c];
    const int gl = threadIdx.x & 15;
    const unsigned int grp = 0xFFFFu << (threadIdx.x & 16);
    NodeCap pc;
    const Geo& G = geo.of(p);
    if (gl == 0) {
        pc = node_cap(G, lvl, pix[p], piy[p]);
        nudge_center(G, lvl, pc, v.pv, v.pe, plist + poff[p], pcnt[p]);
    }
    double P[3];
    P[0] = __shfl_sync(grp, pc.R[0], 0, 16);
    P[1] = __shfl_sync(grp, pc.R[1], 0, 16);
    P[2] = __shfl_sync(grp, pc.R[2], 0, 16);
    const double pr = __shfl_sync(grp, pc.r, 0, 16);
    NodeCap cc;
    {
        const double4 cr = ccaps[c];
        cc.R[0] = cr.x;
        cc.R[1] = cr.y;
        cc.R[2] = cr.z;
        cc.r = ccapsb[c].y;
    }
    if (center_on_vertex(cc.R, v.pv, v.pe, clist + coff[c], ccnt[c])) {
        cc = node_cap(G, lvl + 1, cix[c], ciy[c]);
        nudge_center(G, lvl + 1, cc, v.pv, v.pe, clist + coff[c], ccnt[c]);
    }
    // nesting of caps: the child's cap must lie inside the parent's
    const double dx = P[0] - cc.R[0], dy = P[1] - cc.R[1], dz = P[2] - cc.R[2];
    const double dist = 2.0 * asin(fmin(1.0, 0.5 * sqrt(dx * dx + dy * dy + dz * dz)));
    if (dist + cc.r > pr) atomicAdd(bad + 1, 1);
    const double* Q = cc.R;
    const int* L = plist + poff[p];
    const int n = pcnt[p];
    int par = 0;
    for (int k0 = 0; k0 < n; k0 += 16) {
        int acb_mine = 0;  // -orient(A, B, P) of edge k0 + gl
        if (k0 + gl < n) {
            const int e = L[k0 + gl];
            const D3 a = v.pv[v.pe[2 * e]], b = v.pv[v.pe[2 * e + 1]];
            const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z};
            if (!exact::same(A, B) && !exact::same(A, P) && !exact::same(B, P)) acb_mine = -exact::orient(A, B, P);
        }
        const int m = min(16, n - k0);
        for (int j = 0; j < m; j++) {
            const int acb = __shfl_sync(grp, acb_mine, j, 16);
            const int e = L[k0 + j];
            const D3 a = v.pv[v.pe[2 * e]], b = v.pv[v.pe[2 * e + 1]];
            const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z};
            if (exact::same(A, B)) continue;
            if (exact::same(A, P) || exact::same(B, P) || exact::same(A, Q) || exact::same(B, Q)) {
                atomicAdd(bad, 1);
                continue;
            }
            // exact::crossing(P, Q, A, B) with its first orientation shared
            if (exact::orient(A, B, Q) != acb) continue;
            if (-exact::orient(P, Q, B) != acb) continue;
            if (exact::orient(P, Q, A) == acb) par ^= 1;
        }
    }
    clabel[c] = (uint8_t)(par ? 3 - plabel[p] : plabel[p]);
}

__global__ void k_child_parent(const int* child_base, int np, int cstart, int* child_parent)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np || child_base[p] < 0) return;
    const int b = child_base[p] - cstart;
    for (int k = 0; k < FAN * FAN; k++) child_parent[b + k] = p;
}

// Arc parity against all edges (one arc), with vertex-coincidence flag.
__global__ void k_arc_parity_all(const D3* pv, const int* pe, int n, const double* PQ, int* out)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const D3 a = pv[pe[2 * e]], b = pv[pe[2 * e + 1]];
    const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z};
    if (exact::same(A, B)) return;
    const double* P = PQ;
    const double* Q = PQ + 3;
    if (exact::same(A, P) || exact::same(B, P) || exact::same(A, Q) || exact::same(B, Q)) {
        atomicAdd(out + 1, 1);
        return;
    }
    if (exact::crossing(P, Q, A, B)) {
        atomicXor(out, 1);
        atomicAdd(out + 2, 1);
        atomicMax(out + 3, e);
    }
}

// Final node words, leaf records.
template <class GEO>
__global__ void k_encode(GEO geo, int nn, int gstart, const int* cnt, const int* child_base, const uint8_t* label,
                         const int* leaf_off, uint32_t* nodes)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nn) return;
    uint32_t w;
    if (child_base && child_base[p] >= 0)
        w = KIND_INNER | (uint32_t)(child_base[p] - geo.top(p));
    else if (cnt[p] == 0)
        w = KIND_PURE | label[p];
    else
        w = KIND_LEAF | (uint32_t)leaf_off[p];
    nodes[gstart + p] = w;
}

__global__ void k_leaf_flags(int nn, const int* cnt, const int* child_base, int* is_leaf, int* nrec)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nn) return;
    const bool leaf = cnt[p] > 0 && !(child_base && child_base[p] >= 0);
    is_leaf[p] = leaf ? 1 : 0;
    nrec[p] = leaf ? cnt[p] : 0;
}

template <class GEO>
__global__ void k_leaf_records(BuildView v, GEO geo, int lvl, int nn, const int* is_leaf, const int* leaf_off,
                               const int* rec_off, int leaf_base, long long rec_base, const long long* ix,
                               const long long* iy, const int* cnt, const int* off, const int* list,
                               const uint8_t* label, LeafRec* leaves, float4* recs, uint32_t* eids, double* leafR,
                               int* bad)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nn || !is_leaf[p]) return;
    const Geo& G = geo.of(p);
    NodeCap c = node_cap(G, lvl, ix[p], iy[p]);
    nudge_center(G, lvl, c, v.pv, v.pe, list + off[p], cnt[p]);
    LeafRec L;
    L.lon = c.lonc;
    L.lat = c.latc;
    const long long ro = rec_base + rec_off[p];
    L.off = (uint32_t)ro;
    L.cnt = (uint16_t)min(cnt[p], 65535);
    L.label = label[p];
    L.pad = 0;
    {
        double sb, cb;
        gahhg_canon_sincos(gahhg_canon_rad(L.lat), &sb, &cb);
        L.sb = (float)sb;
        L.cb = (float)cb;
    }
    leaves[leaf_base + leaf_off[p]] = L;
    {
        // the center's canonical XYZ, bit for bit as the query would compute it
        double Rq[3];
        gahhg_canon_vertex_xyz(L.lon, L.lat, Rq);
        double* dst = leafR + 3 * (size_t)(leaf_base + leaf_off[p]);
        dst[0] = Rq[0];
        dst[1] = Rq[1];
        dst[2] = Rq[2];
    }
    if (cnt[p] > 65535) atomicAdd(bad + 2, 1);
    local_frame::Basis fb;
    local_frame::basis_at(c.lonc, c.latc, fb);
    for (int k = 0; k < cnt[p]; k++) {
        const int e = list[off[p] + k];
        const D3 a = v.pv[v.pe[2 * e]], b = v.pv[v.pe[2 * e + 1]];
        const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z};
        const int s1 = exact::orient(A, B, c.R);
        if (s1 == 0) atomicAdd(bad, 1);
        float r[4];
        local_frame::edge_record(A, B, fb, s1 < 0, r);
        recs[ro + k] = make_float4(r[0], r[1], r[2], r[3]);
        eids[ro + k] = (uint32_t)e | (s1 > 0 ? 0x80000000u : 0u);
    }
}

// The FP64 endpoints of every edge side by side, so the FP64 tier reads an
// edge with three aligned 16-byte loads instead of the chain pe -> pv.
__global__ void k_edge_ends(const D3* pv, const int* pe, int n, double2* ends)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const D3 a = pv[pe[2 * e]], b = pv[pe[2 * e + 1]];
    ends[3 * (size_t)e + 0] = make_double2(a.x, a.y);
    ends[3 * (size_t)e + 1] = make_double2(a.z, b.x);
    ends[3 * (size_t)e + 2] = make_double2(b.y, b.z);
}

// Coarse summary of the top level: a coarse cell whose top cells are all
// edge-free with one label gets that label, otherwise "mixed".
__global__ void k_summary(const uint32_t* nodes, int W, int H, int cshift, uint32_t* summary, int ncoarse)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncoarse) return;
    const int f = 1 << cshift;
    const int CW = (W + f - 1) >> cshift;
    const int cx = c % CW, cy = c / CW;
    uint32_t code = 0xFFu;
    for (int y = cy * f; y < min((cy + 1) * f, H) && code != 2u; y++)
        for (int x = cx * f; x < min((cx + 1) * f, W); x++) {
            const uint32_t w = nodes[(size_t)y * W + x];
            const uint32_t v = ((w & KIND_MASK) == KIND_PURE) ? (w & 3u) - 1u : 2u;  // 0 out, 1 in, 2 mixed
            if (code == 0xFFu) code = v;
            else if (code != v) code = 2u;
            if (code == 2u) break;
        }
    atomicOr(&summary[c >> 4], code << ((c & 15) * 2));
}

// Label of the region outside the domain: parity of the arc from a border
// cell's center to the center of the virtual cell just beyond the border
// (both inside the border cell's cap), against that cell's edges.
__global__ void k_outside_label(BuildView v, int ix, int iy, int ox, int oy, const int* cnt, const int* off,
                                const int* list, const uint8_t* label, uint8_t* out, int* bad)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int p = iy * v.g.W + ix;
    NodeCap a = node_cap(v.g, 0, ix, iy);
    nudge_center(v.g, 0, a, v.pv, v.pe, list + off[p], cnt[p]);
    const NodeCap b = node_cap(v.g, 0, ox, oy);
    const int par = arc_parity_lists(v.pv, v.pe, a.R, b.R, list + off[p], cnt[p], nullptr, 0, bad);
    *out = (uint8_t)(par ? 3 - label[p] : label[p]);
}

__global__ void k_shift_leaf_words(uint32_t* nodes, int start, int nn, int add)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nn) return;
    const uint32_t w = nodes[start + p];
    if ((w & KIND_MASK) == KIND_LEAF) nodes[start + p] = w + (uint32_t)add;
}

// ------------------------------------------------------------- query ----

struct QueryView {
    int W, H;
    double Wd, Hd;            // W, H as doubles
    double su_lon, su_lat;    // level-0 cells per degree
    double u0, v0;            // column = lon * su_lon + u0; row = (lat + 90) * su_lat + v0
    double U360;              // cells per 360 degrees of longitude
    int full_lon, to_north, to_south;
    uint32_t outside;         // label outside the domain (pure node word)
    int cshift;               // coarse cell = (1 << cshift) x (1 << cshift) top cells
    int CW;                   // coarse columns
    int swords;               // 32-bit words of the coarse summary
    const uint32_t* summary;  // 2 bits per coarse cell: 0 out, 1 in, 2 mixed
    const uint32_t* nodes;
    const LeafRec* leaves;
    const float4* recs;       // per record: the FP32 tier's tangent-frame ends
    const uint32_t* eids;     // per record: edge id | (orient(A, B, R) > 0) << 31
    const double2* ends;      // per edge: A.xy, A.z B.x, B.yz (48 B, one aligned load each)
    const double* leafR;      // per leaf: the center's canonical XYZ (3 doubles), as leaf_label computes it
    const D3* pv;
    const int* pe;
    int nparts;               // windows of consecutive leaves the pass-2 queue is ordered by (1: none)
    float part_scale;         // window of leaf i: floor(i * part_scale), clamped to nparts - 1
};

struct PointCtx {
    double lon, lat;      // input longitude and FakeLL latitude (canonical XYZ)
    double lon_r, lat_r;  // the same point with lon in [-180, 180], lat in [-90, 90]
    bool have64;
    double q[3];
    __device__ void need64()
    {
        if (!have64) {
            gahhg_canon_vertex_xyz(lon, lat, q);
            have64 = true;
        }
    }
};

// exact sign of orient(x, y, z) given a failed FP32 stage; `code` reports a
// decided label (vertex rule / coincident center) through *early.
__device__ __forceinline__ int sign_escalate(const double* x, const double* y, const double* z,
                                             unsigned long long* cnt64, unsigned long long* cntx)
{
    int s = exact::orient_fp64(x, y, z);
    if (cnt64) atomicAdd(cnt64, 1ull);
    if (s != 0) return s;
    if (cntx) atomicAdd(cntx, 1ull);
    return exact::orient_exact(x, y, z);
}

__device__ uint8_t leaf_label(const QueryView& Q, uint32_t leaf, PointCtx& P, bool fp32, unsigned long long* ctr)
{
    const LeafRec L = Q.leaves[leaf];
    double LR[3];
    gahhg_canon_vertex_xyz(L.lon, L.lat, LR);
    local_frame::Frame f;
    local_frame::Tests ft;
    if (fp32) fp32 = fabs(P.lon) <= 540.0 && local_frame::frame_at(P.lon, P.lat, L.lon, L.lat, L.sb, L.cb, f);
    if (fp32) local_frame::tests_of(f, ft);
    if (!fp32) P.need64();
    unsigned long long* c64 = ctr ? ctr + 0 : nullptr;
    unsigned long long* cx = ctr ? ctr + 1 : nullptr;
    int par = 0;
    for (int k = 0; k < L.cnt; k++) {
        const uint32_t es = __ldg(Q.eids + L.off + k);
        const int e = (int)(es & 0x7fffffffu);
        const int s1 = (es >> 31) ? 1 : -1;
        // the record holds (A, B) when s1 = +1, else (B, A): see local_frame.cuh
        int s2 = 0, ea = 0, eb = 0;
        if (fp32) {
            const float4 r = __ldg(Q.recs + L.off + k);
            s2 = s1 * local_frame::sign_edge(ft, r.x, r.y, r.z, r.w);
            const float x1 = s1 > 0 ? r.x : r.z, x2 = s1 > 0 ? r.y : r.w;
            const float y1 = s1 > 0 ? r.z : r.x, y2 = s1 > 0 ? r.w : r.y;
            ea = local_frame::sign_end(ft, x1, x2);
            eb = local_frame::sign_end(ft, y1, y2);
        }
        double A[3], B[3];
        bool haveAB = false;
        auto needAB = [&]() {
            if (!haveAB) {
                const D3 a = Q.pv[Q.pe[2 * e]], b = Q.pv[Q.pe[2 * e + 1]];
                A[0] = a.x;
                A[1] = a.y;
                A[2] = a.z;
                B[0] = b.x;
                B[1] = b.y;
                B[2] = b.z;
                haveAB = true;
            }
        };
        if (s2 == 0) {
            P.need64();
            needAB();
            if (exact::same(P.q, A) || exact::same(P.q, B)) return CELL_IN;  // vertex rule
            if (exact::same(P.q, LR)) return L.label;                       // q is the center
            s2 = sign_escalate(A, B, P.q, c64, cx);
        }
        if (s2 == s1) continue;
        // s3 = orient(R, q, A); crossing needs s3 == s2
        int s3 = ea;
        if (s3 == 0) {
            P.need64();
            needAB();
            if (exact::same(P.q, A) || exact::same(P.q, B)) return CELL_IN;
            if (exact::same(P.q, LR)) return L.label;
            s3 = sign_escalate(LR, P.q, A, c64, cx);
        }
        if (s3 != s2) continue;
        int s4 = eb;
        if (s4 == 0) {
            P.need64();
            needAB();
            if (exact::same(P.q, A) || exact::same(P.q, B)) return CELL_IN;
            if (exact::same(P.q, LR)) return L.label;
            s4 = sign_escalate(LR, P.q, B, c64, cx);
        }
        if (s4 == -s2) par ^= 1;
    }
    return (uint8_t)(par ? 3 - L.label : L.label);
}

// Programmatic dependent launch (sm_90+): a kernel launched with
// programmatic stream serialization may start while its predecessor drains;
// it waits here until the predecessor's grid has completed and its memory is
// visible.  Predecessors allow the start when a block has finished its main
// loop: allowing it at their beginning made the waiting blocks of the next
// tier hold registers through the whole pass (14 % slower on near-edge
// points), allowing it at the end only hides the launch of the next tier.
__device__ __forceinline__ void wait_for_predecessor() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allow_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// ------------------------------------------- summary staging by bulk copy --
//
// The coarse summary (up to 16 KB) goes to shared memory by one bulk copy
// (TMA, untiled cp.async.bulk global -> shared, completion counted on an
// mbarrier in bytes; no multicast) issued by one thread, instead of a load
// per word by every thread.  Both addresses are 16-byte aligned (pool
// allocations are 256-byte aligned, the shared arrays are declared so) and
// the size is rounded up to 16 bytes (the summary's allocation holds at least
// 1,024 words).  Every wait is bounded; a wait that runs out is counted in
// g_tma_timeouts and the block falls back to loading the summary itself into
// memory no pending copy can write (see the kernels), so labels never depend
// on a copy completing.

__device__ unsigned int g_tma_timeouts;
constexpr int MBAR_POLL_LIMIT = 1 << 20;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One thread: the copy of `bytes` from global `src` to shared `dst`,
// completing the barrier's current phase.
__device__ __forceinline__ void bulk_stage(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    // earlier generic-proxy reads of dst (ordered by the block barrier) come
    // before the async-proxy write
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Bounded wait for the phase with the given parity; false when it ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit = MBAR_POLL_LIMIT)
{
    for (int i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__host__ __device__ __forceinline__ uint32_t summary_bytes(int swords) { return ((uint32_t)swords * 4u + 15u) & ~15u; }

// ------------------------------------------------------ escalation tiers --
//
// The crossing tests of the queued points run in tiers, each its own launch
// over the points the previous tier could not decide, so that no warp carries
// the registers or waits on the branches of a rarer, costlier tier:
//   tier 1: every sign from the certified FP32 filter in the leaf's local
//           frame (local_frame.cuh);
//   tier 2: the canonical FP64 point, the vertex and center rules, and every
//           sign from the FP64 filter on translated rows (orient_fp64_near);
//   tier 3: the complete test (FP64 filter, then exact arithmetic with
//           simulation of simplicity), leaf_label above.
// Every sign a tier returns is exact, so a label does not depend on the tier
// that produced it.
constexpr uint8_t LABEL_DEFER = 0xFF;

// Tier 1 runs every edge of the leaf: a decided edge adds its crossing to
// the parity, an undecided one is noted in `mask` (bit k for record k < 31)
// and the FP64 tier evaluates only those, starting from the parity of the
// decided ones (bit 31).  The label is exact either way: the crossing parity
// is the XOR of independent per-edge tests.  MASK_ALL asks tier 2 for every
// edge (a record beyond the 31st undecided, or the offset refused).
constexpr uint32_t MASK_ALL = 0xFFFFFFFFu;

// Records whose loads tier 1 issues together (one group covers a leaf of
// the default leaf size): the first group goes out before the offset's
// arithmetic, so its latency hides behind the sines and cosines.
constexpr int T1_GROUP = 4;
// Blocks per SM of tier 1: five (48 registers, 20 bytes spilled) ran C2 at
// 21.0-21.1 Gpts/s against 20.5 at four (56 registers); five with groups of
// two (no spills) 20.5, six with groups of two (40 registers) 20.8.
constexpr int T1_BLOCKS = 5;

// A record of tier 1: from global memory through the read-only path, or
// from a copy in shared memory (SHARED).
template <bool SHARED>
__device__ __forceinline__ float4 t1_record(const float4* p)
{
    if constexpr (SHARED) return *p;
    else return __ldg(p);
}

// Tier 1 on the leaf L whose records start at rec (global memory, or the
// staged copy in shared memory when SHARED).
template <bool SHARED>
__device__ __forceinline__ uint8_t leaf_label_fp32_at(const float4* rec, const LeafRec& L, const PointCtx& P,
                                                    uint32_t& mask)
{
    const int cnt = L.cnt;
    float4 r[T1_GROUP];
#pragma unroll
    for (int j = 0; j < T1_GROUP; j++) r[j] = j < cnt ? t1_record<SHARED>(rec + j) : make_float4(0.f, 0.f, 0.f, 0.f);
    local_frame::Frame f;
    if (!(fabs(P.lon) <= 540.0) || !local_frame::frame_at(P.lon, P.lat, L.lon, L.lat, L.sb, L.cb, f)) {
        mask = MASK_ALL;
        return LABEL_DEFER;
    }
    local_frame::Tests t;
    local_frame::tests_of(f, t);
    int par = 0;
    uint32_t und = 0;
    bool all = false;
    for (int k0 = 0; k0 < cnt; k0 += T1_GROUP) {
        if (k0 > 0) {
#pragma unroll
            for (int j = 0; j < T1_GROUP; j++)
                r[j] = k0 + j < cnt ? t1_record<SHARED>(rec + k0 + j) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int j = 0; j < T1_GROUP; j++) {
            const int k = k0 + j;
            if (k >= cnt) break;
            const int x = local_frame::record_crossing(t, r[j].x, r[j].y, r[j].z, r[j].w);
            if (x > 0) par ^= 1;
            if (x < 0) {
                if (k < 31)
                    und |= 1u << k;
                else
                    all = true;
            }
        }
    }
    if (all) {
        mask = MASK_ALL;
        return LABEL_DEFER;
    }
    if (und) {
        mask = und | ((uint32_t)par << 31);
        return LABEL_DEFER;
    }
    return (uint8_t)(par ? 3 - L.label : L.label);
}

__device__ __forceinline__ uint8_t leaf_label_fp32(const QueryView& Q, const LeafRec& L, const PointCtx& P,
                                                 uint32_t& mask)
{
    return leaf_label_fp32_at<false>(Q.recs + L.off, L, P, mask);
}

// Edges of a leaf whose FP64 endpoints the FP64 tier loads together: their
// loads (edge id, then three 16-byte loads of the endpoints) are all in flight
// before the first sign is evaluated, instead of one dependent chain per edge.
constexpr int T2_GROUP = 4;

// FP64 tier on the leaf's records selected by `mask` (MASK_ALL: every record,
// parity from 0; else the records of bits 0..30, parity from bit 31).
__device__ uint8_t leaf_label_fp64(const QueryView& Q, uint32_t leaf, PointCtx& P, uint32_t mask = MASK_ALL)
{
    const LeafRec L = Q.leaves[leaf];
    // the leaf's loads go out before the point's canonical XYZ is computed
    const double LR[3] = {__ldg(Q.leafR + 3 * (size_t)leaf), __ldg(Q.leafR + 3 * (size_t)leaf + 1),
                          __ldg(Q.leafR + 3 * (size_t)leaf + 2)};
    const bool all = mask == MASK_ALL;
    const int cnt = L.cnt;
    int par = all ? 0 : (int)(mask >> 31);
    uint32_t sel = all ? 0u : (mask & 0x7fffffffu);
    int kk[T2_GROUP];
    uint32_t es[T2_GROUP];
    // the next T2_GROUP records (consecutive ones, or the next set bits of
    // sel) and their edge words
    auto next_group = [&](int k0) {
#pragma unroll
        for (int j = 0; j < T2_GROUP; j++) {
            if (all) {
                kk[j] = k0 + j < cnt ? k0 + j : -1;
            } else if (sel) {
                kk[j] = __ffs(sel) - 1;
                sel &= sel - 1u;
            } else {
                kk[j] = -1;
            }
        }
#pragma unroll
        for (int j = 0; j < T2_GROUP; j++) es[j] = kk[j] >= 0 ? __ldg(Q.eids + L.off + kk[j]) : 0u;
    };
    // the first group's edge words are in flight while the point's canonical
    // XYZ is computed
    next_group(0);
    P.need64();
    for (int k0 = 0; kk[0] >= 0; k0 += T2_GROUP) {
        double2 e[T2_GROUP][3];
#pragma unroll
        for (int j = 0; j < T2_GROUP; j++) {
            if (kk[j] >= 0) {
                const double2* p = Q.ends + 3 * (size_t)(es[j] & 0x7fffffffu);
                e[j][0] = __ldg(p);
                e[j][1] = __ldg(p + 1);
                e[j][2] = __ldg(p + 2);
            }
        }
#pragma unroll
        for (int j = 0; j < T2_GROUP; j++) {
            if (kk[j] < 0) break;
            const int s1 = (es[j] >> 31) ? 1 : -1;
            const double A[3] = {e[j][0].x, e[j][0].y, e[j][1].x}, B[3] = {e[j][1].y, e[j][2].x, e[j][2].y};
            if (exact::same(P.q, A) || exact::same(P.q, B)) return CELL_IN;  // vertex rule
            if (exact::same(P.q, LR)) return L.label;                       // q is the center
            // every row is within a cap of the first: translated rows keep the bound small
            const int s2 = exact::orient_fp64_near(A, B, P.q);
            if (s2 == 0) return LABEL_DEFER;
            if (s2 == s1) continue;
            const int s3 = exact::orient_fp64_near(LR, P.q, A);
            if (s3 == 0) return LABEL_DEFER;
            if (s3 != s2) continue;
            const int s4 = exact::orient_fp64_near(LR, P.q, B);
            if (s4 == 0) return LABEL_DEFER;
            if (s4 == -s2) par ^= 1;
        }
        if (all ? k0 + T2_GROUP >= cnt : sel == 0u) break;
        next_group(k0 + T2_GROUP);
    }
    return (uint8_t)(par ? 3 - L.label : L.label);
}

// Level-0 cell of a point from its longitude and FakeLL latitude + 90
// (`laf`); false when the point lies outside the domain.
struct Loc {
    int ix, iy;
    double fu, fv;
};

// Level-0 cell of a point from its longitude and FakeLL latitude + 90
// (`laf`); false when the point lies outside the domain.  Inside the domain
// this costs two multiply-adds, two conversions and two unsigned compares;
// points beyond a non-polar latitude edge are rejected with one more compare.
__device__ __forceinline__ bool domain_locate(const QueryView& Q, double lo, double laf, Loc& L)
{
    double u = fma(lo, Q.su_lon, Q.u0), v = fma(laf, Q.su_lat, Q.v0);
    int ix = __double2int_rd(u), iy = __double2int_rd(v);
    if ((unsigned)iy >= (unsigned)Q.H) {
        if (iy < 0 ? !Q.to_south : !Q.to_north) return false;
        // a domain that reaches the pole keeps the pole in its first/last row
        const bool below = iy < 0;
        iy = below ? 0 : Q.H - 1;
        v = below ? 0.0 : fmin(v, Q.Hd);
    }
    if ((unsigned)ix >= (unsigned)Q.W) {
        if (u < 0.0) u += Q.U360;
        if (u < 0.0) u += Q.U360;
        if (u >= Q.U360) u -= Q.U360;
        if (u >= Q.U360) u -= Q.U360;
        ix = __double2int_rd(u);
        if ((unsigned)ix >= (unsigned)Q.W) {
            if (!Q.full_lon) return false;
            ix = ix < 0 ? 0 : Q.W - 1;
        }
    }
    L.ix = ix;
    L.iy = iy;
    L.fu = u - ix;
    L.fv = v - iy;
    return true;
}

// A cell fraction in [0, 1) as a 32-bit binary fraction, saturating (below 0
// gives 0, 1 and above all ones).  Its base-4 digits are the children that
// the recursion f -> 4 f - floor(4 f) (clamped to 0..3) visits: that FP64
// recursion is exact, so digit k of the fraction is its k-th child for the
// first 16 levels, and for the clamped out-of-range cases both give 0 or 3 at
// every level.  The lattice has at most MAX_DESCENT levels below the top.
constexpr int MAX_DESCENT = 16;
__device__ __forceinline__ uint32_t frac_bits(double f) { return __double2uint_rz(f * 4294967296.0); }

__device__ __forceinline__ uint32_t descend(const QueryView& Q, uint32_t w, double fu, double fv)
{
    uint32_t U = frac_bits(fu), V = frac_bits(fv);
    while ((w & KIND_MASK) == KIND_INNER) {
        w = __ldg(Q.nodes + (w & INDEX_MASK) + (V >> 30) * FAN + (U >> 30));
        U <<= 2;
        V <<= 2;
    }
    return w;
}

// block-reduced count of inside labels (statistics only)
__device__ __forceinline__ void count_inside(int v, unsigned long long* dst)
{
    __shared__ int s_sum;
    if (threadIdx.x == 0) s_sum = 0;
    __syncthreads();
    for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xffffffffu, v, d);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&s_sum, v);
    __syncthreads();
    if (threadIdx.x == 0 && s_sum) atomicAdd(dst, (unsigned long long)s_sum);
}

constexpr int LOC_UNROLL = 4;
constexpr uint8_t LABEL_PENDING = 0;
// Leaf word of a queued point that pass 1 did not locate (a pure node
// without a label, which is never queued).
constexpr uint32_t LEAF_UNKNOWN = KIND_PURE;

// Pass 1: every point whose cell has no edges gets its label; the others are
// queued (index within this chunk) for pass 2.  Lean on registers and
// instructions so that many warps keep loads in flight; lon/lat and labels
// stream with an evict-first policy so the node table stays in L2.  The index
// arithmetic need not match the canonical conversion bit for bit: every cap
// carries a margin far above its rounding (see LOC_MARGIN).
// Pass 1 over points [first, first + count) of one polygon, in tiles of
// TPB * LOC_UNROLL points (tiles tile0, tile0 + tstride, ...): every point
// whose cell has no edges gets its label; the others are queued (their index
// `first + local`) for pass 2.  Lean on registers and instructions so that
// many warps keep loads in flight; lon/lat and labels stream with an
// evict-first policy so the node table stays in L2.  The index arithmetic
// need not match the canonical conversion bit for bit: every cap carries a
// margin far above its rounding (see LOC_MARGIN).
template <bool STATS, bool LOCKSTEP = false, int UNROLL = LOC_UNROLL>
__device__ __forceinline__ void locate_range(const QueryView& Q, const uint32_t* s_sum,
                                             const double2* __restrict__ ll, uint8_t* __restrict__ out,
                                             uint32_t* __restrict__ queue, uint32_t* __restrict__ leafq,
                                             unsigned int* __restrict__ qcount, long long first, int count,
                                             int tile0, int tstride, int& inside)
{
    const int lane = threadIdx.x & 31;
    const int cs = Q.cshift, cw = Q.CW;
    constexpr int TILE = TPB * UNROLL;
    for (int base = tile0 * TILE; base < count; base += tstride * TILE) {
        const bool full = base + TILE <= count;
        double2 p[UNROLL];
#pragma unroll
        for (int k = 0; k < UNROLL; k++) {
            const int i = base + k * TPB + threadIdx.x;
            p[k] = (full || i < count) ? __ldcs(ll + first + i) : make_double2(0.0, 0.0);
        }
        uint8_t lab[UNROLL];
        bool push[UNROLL];
        bool any = false;
        // LOCKSTEP: the node words of all points are loaded first and the
        // descents advance one level per round, so a thread keeps one
        // independent load per point in flight (points that mostly need the
        // node table, as around small polygons, are bound by its latency)
        uint32_t w[UNROLL];
        uint32_t fu[UNROLL], fv[UNROLL];  // cell fractions as binary fractions (frac_bits)
#pragma unroll
        for (int k = 0; k < UNROLL; k++) {
            const int i = base + k * TPB + threadIdx.x;
            const double lo = p[k].x;
            const double laf = p[k].y + 90.0;  // the reference's FakeLL latitude + 90
            lab[k] = LABEL_PENDING;
            push[k] = false;
            w[k] = KIND_PURE;
            if (full || i < count) {
                if (laf >= 0.0 && laf <= 180.0 && fabs(lo) <= 540.0) {
                    Loc L;
                    if (!domain_locate(Q, lo, laf, L)) {
                        lab[k] = (uint8_t)Q.outside;
                    } else {
                        const int c = (L.iy >> cs) * cw + (L.ix >> cs);
                        const uint32_t code = (s_sum[c >> 4] >> ((c & 15) << 1)) & 3u;
                        if (code < 2u) {
                            lab[k] = (uint8_t)(code + 1u);  // coarse cell without edges: most points end here
                        } else if (LOCKSTEP) {
                            w[k] = __ldg(Q.nodes + (size_t)L.iy * Q.W + L.ix);
                            fu[k] = frac_bits(L.fu);
                            fv[k] = frac_bits(L.fv);
                        } else {
                            const uint32_t d = descend(Q, __ldg(Q.nodes + (size_t)L.iy * Q.W + L.ix), L.fu, L.fv);
                            if ((d & KIND_MASK) == KIND_PURE)
                                lab[k] = (uint8_t)(d & 3u);
                            else
                                push[k] = true;
                            w[k] = d;
                        }
                    }
                } else {
                    // unusual coordinates go to pass 2; non-finite input stays undefined
                    push[k] = isfinite(lo) && isfinite(laf);
                }
            }
            if (!LOCKSTEP) any |= push[k];
        }
        if (LOCKSTEP) {
            bool inner = true;
            while (inner) {
                inner = false;
#pragma unroll
                for (int k = 0; k < UNROLL; k++)
                    if ((w[k] & KIND_MASK) == KIND_INNER) {
                        w[k] = __ldg(Q.nodes + (w[k] & INDEX_MASK) + (fv[k] >> 30) * FAN + (fu[k] >> 30));
                        fu[k] <<= 2;
                        fv[k] <<= 2;
                        inner = true;
                    }
            }
#pragma unroll
            for (int k = 0; k < UNROLL; k++) {
                if (lab[k] == LABEL_PENDING && !push[k]) {
                    const int i = base + k * TPB + threadIdx.x;
                    if (full || i < count) {
                        if ((w[k] & KIND_MASK) == KIND_PURE) {
                            if (w[k] != KIND_PURE) lab[k] = (uint8_t)(w[k] & 3u);  // KIND_PURE alone: no node read
                        } else {
                            push[k] = true;
                        }
                    }
                }
                any |= push[k];
            }
        }
        if (__any_sync(0xffffffffu, any)) {
            // one atomic on the queue counter per warp and tile: every thread of
            // the grid pushes through this one counter, and where most points
            // are queued (points near the edges) the counter itself limits pass 1
            // (one per block and tile, which takes block-wide barriers, made
            // uniform points 14 % slower and near-edge points 2 % faster)
            unsigned int total = 0;
#pragma unroll
            for (int k = 0; k < UNROLL; k++) total += __popc(__ballot_sync(0xffffffffu, push[k]));
            unsigned int pos = 0;
            if (lane == 0) pos = atomicAdd(qcount, total);
            pos = __shfl_sync(0xffffffffu, pos, 0);
#pragma unroll
            for (int k = 0; k < UNROLL; k++) {
                const unsigned int mk = __ballot_sync(0xffffffffu, push[k]);
                if (push[k]) {
                    const unsigned int at = pos + __popc(mk & ((1u << lane) - 1u));
                    queue[at] = (uint32_t)(first + base + k * TPB + threadIdx.x);
                    // w is the leaf word, or KIND_PURE (LEAF_UNKNOWN) for an unlocated point
                    if (leafq) leafq[at] = w[k];
                }
                pos += __popc(mk);
            }
        }
#pragma unroll
        for (int k = 0; k < UNROLL; k++) {
            const int i = base + k * TPB + threadIdx.x;
            if (full || i < count) __stcs(out + first + i, lab[k]);
            if (STATS) inside += lab[k] == CELL_IN;
        }
    }
}

template <bool STATS>
__global__ void __launch_bounds__(TPB) k_locate(const double2* __restrict__ ll, int n, uint8_t* __restrict__ out,
                                               QueryView Q, uint32_t* __restrict__ queue,
                                               uint32_t* __restrict__ leafq, unsigned int* __restrict__ qcount,
                                               unsigned long long* ctr, int poll_limit)
{
    extern __shared__ __align__(16) uint32_t s_sum[];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ int s_late;
    if (threadIdx.x == 0) {
        s_late = 0;
        mbar_init(&s_bar);
        bulk_stage(s_sum, Q.summary, summary_bytes(Q.swords), &s_bar);
    }
    __syncthreads();
    if (!mbar_wait(&s_bar, 0, poll_limit)) s_late = 1;
    __syncthreads();
    const bool late = s_late != 0;
    // after a wait that ran out the block reads the summary from global
    // memory and never touches s_sum, which the pending copy still targets
    if (late && threadIdx.x == 0) atomicAdd(&g_tma_timeouts, 1u);
    int inside = 0;
    locate_range<STATS>(Q, late ? Q.summary : s_sum, ll, out, queue, leafq, qcount, 0, n, blockIdx.x, gridDim.x,
                        inside);
    if (late) mbar_wait(&s_bar, 0);  // the copy in flight ends before the block does (bounded)
    allow_dependents();
    if (STATS && ctr) count_inside(inside, ctr + 3);
}

// The leaf of a queued point (the point context filled in), or its label
// with KIND_PURE when its cell has no edges.
// The point's context, and its node word: `known` when pass 1 located the
// point (any leaf it finds serves: every leaf cap holds its points with a
// margin above the locate arithmetic's rounding), else a descent from the top.
__device__ __forceinline__ uint32_t point_leaf(const QueryView& Q, double2 p, PointCtx& P,
                                              uint32_t known = LEAF_UNKNOWN)
{
    P.lat = gahhg_canon_query_lat(p.y);
    P.lon = p.x;
    P.have64 = false;
    double lo = P.lon, la = P.lat;
    if (!(fabs(lo) <= 540.0 && fabs(la) <= 90.0)) {
        // unusual input: locate from the canonical XYZ itself
        P.need64();
        la = asin(fmin(1.0, fmax(-1.0, P.q[1]))) / RAD;
        lo = atan2(P.q[0], P.q[2]) / RAD;
    }
    Loc L;
    double lr = lo;
    if (lr > 180.0) lr -= 360.0;
    if (lr > 180.0) lr -= 360.0;
    if (lr < -180.0) lr += 360.0;
    if (lr < -180.0) lr += 360.0;
    P.lon_r = lr;
    P.lat_r = la;
    if (known != LEAF_UNKNOWN) return known;
    const bool in = domain_locate(Q, lo, la + 90.0, L);
    return in ? descend(Q, __ldg(Q.nodes + (size_t)L.iy * Q.W + L.ix), L.fu, L.fv) : Q.outside;
}

// One point through the untiered path (escalations inline, counted per test).
template <bool FP32>
__device__ __forceinline__ uint8_t leaf_point(const QueryView& Q, double2 p, unsigned long long* ctr)
{
    PointCtx P;
    const uint32_t w = point_leaf(Q, p, P);
    if ((w & KIND_MASK) == KIND_PURE) return (uint8_t)(w & 3u);
    if (ctr) atomicAdd(ctr + 2, 1ull);
    return leaf_label(Q, w & INDEX_MASK, P, FP32, ctr);
}

// Pass 2: exact crossing tests for the queued points.
template <bool FP32>
__global__ void __launch_bounds__(TPB) k_leaf(const double2* __restrict__ ll, uint8_t* __restrict__ out,
                                             QueryView Q, const uint32_t* __restrict__ queue,
                                             const unsigned int* __restrict__ qcount, unsigned long long* ctr)
{
    const unsigned int m = *qcount;
    int inside = 0;
    for (unsigned int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
        const uint32_t i = queue[t];
        const uint8_t lab = leaf_point<FP32>(Q, ll[i], ctr);
        out[i] = lab;
        inside += lab == CELL_IN;
    }
    if (ctr) count_inside(inside, ctr + 3);
}

// ------------------------------------------------------------- batches --

// A run of points of one view (points are stored segment after segment, and
// chunks are in point order, so chunk starts are increasing).
struct BatchChunk {
    int view;
    int count;
    long long start;
};

constexpr int BATCH_SUMMARY_WORDS = 4096;  // 16 KB of shared memory
// Launch shapes of the batch locate: points per thread in flight (in
// lockstep) and blocks per SM (all resident; each holds 32 KB of shared
// memory, and the register budget per thread follows from the blocks).  The
// default, five points at five blocks (48 registers), took a 1,024-polygon
// C3 batch from 75.6 (8 points, two blocks) to 106.5 Gpts/s; 4 x 5 101.2,
// 6 x 4 101.8, 6 x 5 102.3, 4 x 6 91.2, 8 x 3 93.5 (labels identical): more
// warps hide more of the node descents' latency than more points per
// thread (2 x 6 spills at 40 registers and ran at 56.6).  Batches of other
// point mixes may prefer another row (4 x 4 leaves fewer lanes idle in
// chunks of few points); the batch autotuner measures them.
struct BatchShape {
    int unroll, blocks;
};
constexpr BatchShape BATCH_SHAPES[] = {{5, 5}, {4, 4}, {6, 4}, {8, 3}};
constexpr int BATCH_NSHAPES = (int)(sizeof(BATCH_SHAPES) / sizeof(BATCH_SHAPES[0]));

// Pass 1 over a batch: a persistent grid takes chunks in order from an atomic
// counter (polygons of very different sizes balance themselves), stages the
// chunk's polygon summary in shared memory and runs the single-polygon tile
// loop on it.
template <bool STATS, int UNROLL, int BLOCKS>
__global__ void __launch_bounds__(TPB, BLOCKS) k_batch_locate(const QueryView* __restrict__ views,
                                                     const BatchChunk* __restrict__ chunks, int nchunks,
                                                     unsigned int* next_chunk, const double2* __restrict__ ll,
                                                     uint8_t* __restrict__ out, uint32_t* __restrict__ queue,
                                                     uint32_t* __restrict__ leafq, unsigned int* __restrict__ qcount,
                                                     unsigned long long* ctr, int poll_limit)
{
    // s_sum receives the bulk copies; after a wait runs out the block loads
    // summaries itself into s_own, which no copy writes
    __shared__ __align__(16) uint32_t s_sum[BATCH_SUMMARY_WORDS];
    __shared__ __align__(16) uint32_t s_own[BATCH_SUMMARY_WORDS];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ int s_chunk, s_late;
    if (threadIdx.x == 0) {
        s_late = 0;
        mbar_init(&s_bar);
    }
    uint32_t phase = 0;
    bool late = false;  // the same in every thread: read from s_late after a barrier
    int inside = 0;
    for (;;) {
        if (threadIdx.x == 0) s_chunk = (int)atomicAdd(next_chunk, 1u);
        __syncthreads();
        const int ci = s_chunk;
        if (ci >= nchunks) break;
        const BatchChunk c = chunks[ci];
        const QueryView Q = views[c.view];
        const uint32_t* sum = s_sum;
        if (!late) {
            if (threadIdx.x == 0) bulk_stage(s_sum, Q.summary, summary_bytes(Q.swords), &s_bar);
            if (!mbar_wait(&s_bar, phase, poll_limit)) s_late = 1;  // any thread's timeout switches the block
            phase ^= 1u;
            __syncthreads();
            late = s_late != 0;
        }
        if (late) {
            for (int k = threadIdx.x; k < Q.swords; k += TPB) s_own[k] = __ldg(Q.summary + k);
            sum = s_own;
            __syncthreads();
        }
        locate_range<STATS, true, UNROLL>(Q, sum, ll, out, queue, leafq, qcount, c.start, c.count, 0, 1, inside);
        __syncthreads();
    }
    if (late) {
        if (threadIdx.x == 0) atomicAdd(&g_tma_timeouts, 1u);
        mbar_wait(&s_bar, phase ^ 1u);  // the copy in flight ends before the block does (bounded)
    }
    allow_dependents();
    if (STATS && ctr) count_inside(inside, ctr + 3);
}

// Escalation queues of one pass-2 run.  cnt[0] / cnt[1] count the points
// deferred to tier 2 / tier 3 (they keep counting past the capacities);
// cnt[2] is raised when a point found its queue full: it stays unlabelled
// (pass 1 wrote LABEL_PENDING) and the final sweep gives it the complete
// test, so no tier carries the code of the tiers after it.
// Every queue of points has a parallel array of leaf words (l1 for the
// pass-1 queue): the node word pass 1 found for the point, or LEAF_UNKNOWN
// when it did not locate it, so the tiers need not descend again.
struct Tiers {
    uint32_t* q2;
    uint32_t* q3;
    uint32_t* l1;
    uint32_t* l2;
    uint32_t* l3;
    uint32_t* m2;   // per tier-2 entry: tier 1's mask of undecided records (leaf_label_fp32)
    unsigned int* cnt;
    unsigned int cap2, cap3;
    // the pass-1 queue in window order (k_part_scatter), used by the first
    // tier when *sorted == 1
    const uint32_t* spts = nullptr;
    const uint32_t* sleaf = nullptr;
    const unsigned int* sorted = nullptr;
    int sstride = 1;  // words from one ordered entry to the next (2: leaf order's interleaved pairs)
};

// The pass-1 queue as the first tier reads it: in window order when
// k_part_scatter ran, else in pass-1 order.
__device__ __forceinline__ void first_tier_source(const Tiers& T, const uint32_t*& pts, const uint32_t*& leaf,
                                                  unsigned int& stride)
{
    stride = 1;
    if (T.sorted && *(const volatile unsigned int*)T.sorted == 1u) {
        pts = T.spts;
        leaf = T.sleaf;
        stride = (unsigned int)T.sstride;
    }
}

// Where a queued point's index view comes from: one polygon...
struct OneView {
    QueryView Q;
    __device__ __forceinline__ const QueryView& of(uint32_t) const { return Q; }
};

// ...or the chunk holding it (binary search of the chunk starts).
struct ChunkViews {
    const QueryView* views;
    const BatchChunk* chunks;
    int nchunks;
    __device__ __forceinline__ const QueryView& of(uint32_t i) const
    {
        int lo = 0, hi = nchunks;  // chunks[lo].start <= i < chunks[hi].start
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (__ldg(&chunks[mid].start) <= (long long)i) lo = mid;
            else hi = mid;
        }
        return views[__ldg(&chunks[lo].view)];
    }
};

// Appends i to q through counter *c, one atomic per group of converged
// threads; false when the queue is full.
__device__ __forceinline__ bool push_deferred(uint32_t i, uint32_t w, uint32_t* q, uint32_t* l, unsigned int* c,
                                              unsigned int cap, uint32_t* extra = nullptr, uint32_t x = 0u)
{
    const unsigned int act = __activemask();
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(act) - 1;
    unsigned int base = 0;
    if (lane == leader) base = atomicAdd(c, (unsigned int)__popc(act));
    base = __shfl_sync(act, base, leader);
    const unsigned int pos = base + __popc(act & ((1u << lane) - 1u));
    if (pos >= cap) return false;
    q[pos] = i;
    l[pos] = w;
    if (extra) extra[pos] = x;
    return true;
}

__device__ __forceinline__ void count_stats(unsigned long long* ctr, int inside, int boundary, int fp64, int exact)
{
    count_inside(inside, ctr + 3);
    count_inside(boundary, ctr + 2);
    count_inside(fp64, ctr + 0);
    count_inside(exact, ctr + 1);
}

// Tier 1 over the pass-1 queue.
template <class VS>
__global__ void __launch_bounds__(TPB, T1_BLOCKS) k_leaf_t1(VS vs, const double2* __restrict__ ll,
                                                         uint8_t* __restrict__ out, const uint32_t* __restrict__ queue,
                                                         const unsigned int* __restrict__ qcount, Tiers T,
                                                         unsigned long long* ctr)
{
    __shared__ unsigned int s_wcnt[TPB / 32];
    __shared__ unsigned int s_base;
    wait_for_predecessor();
    const unsigned int m = *qcount;
    const uint32_t* src = queue;
    const uint32_t* src_leaf = T.l1;
    unsigned int st;
    first_tier_source(T, src, src_leaf, st);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inside = 0, boundary = 0, fp64 = 0;
    // block-uniform loop: the deferred points of a block's round take one
    // atomic on the tier-2 counter (about half the points defer on near-edge
    // inputs, and one counter serves the whole grid)
    for (unsigned int b0 = blockIdx.x * blockDim.x; b0 < m; b0 += gridDim.x * blockDim.x) {
        const unsigned int t = b0 + threadIdx.x;
        bool defer = false;
        uint32_t i = 0, w = 0, mask = 0;
        if (t < m) {
            i = src[t * st];
            const uint32_t known = src_leaf[t * st];
            const QueryView& Q = vs.of(i);
            // the leaf record (a point pass 1 located in a leaf) is loaded
            // with the point's coordinates, not after them
            const bool in_leaf = (known & KIND_MASK) == KIND_LEAF;
            LeafRec L0;
            if (in_leaf) L0 = Q.leaves[known & INDEX_MASK];
            PointCtx P;
            w = point_leaf(Q, ll[i], P, known);
            uint8_t lab;
            if ((w & KIND_MASK) == KIND_PURE) {
                lab = (uint8_t)(w & 3u);
            } else {
                boundary++;
                lab = leaf_label_fp32(Q, in_leaf ? L0 : Q.leaves[w & INDEX_MASK], P, mask);
            }
            if (lab == LABEL_DEFER) {
                fp64++;
                defer = true;
            } else {
                out[i] = lab;
                inside += lab == CELL_IN;
            }
        }
        const unsigned int bal = __ballot_sync(0xffffffffu, defer);
        if (lane == 0) s_wcnt[warp] = __popc(bal);
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned int tot = 0;
            for (int k = 0; k < TPB / 32; k++) {
                const unsigned int c = s_wcnt[k];
                s_wcnt[k] = tot;
                tot += c;
            }
            s_base = tot ? atomicAdd(T.cnt, tot) : 0u;
        }
        __syncthreads();
        if (defer) {
            const unsigned int pos = s_base + s_wcnt[warp] + __popc(bal & ((1u << lane) - 1u));
            if (pos < T.cap2) {
                T.q2[pos] = i;
                T.l2[pos] = w;
                T.m2[pos] = mask;
            } else {
                T.cnt[2] = 1;  // the tier-3 sweep labels it
            }
        }
        __syncthreads();  // s_wcnt / s_base are rewritten next round
    }
    allow_dependents();
    if (ctr) count_stats(ctr, inside, boundary, fp64, 0);
}

// ---------------------------------- tier 1 with the edge lists staged --
//
// Over the pass-1 queue in leaf order (k_ls_*), the entries of a tile of TPB
// consecutive entries lie in a run of consecutive leaves, and leaves are
// numbered so that their records are contiguous: the tile's leaf records and
// the edge records of those leaves are two contiguous slices of the index.
// One thread copies both into shared memory (TMA: two untiled cp.async.bulk
// global -> shared, completion counted in bytes on one mbarrier; no
// multicast, the source is this GPU's index) while the block loads its
// points and their frames, and every crossing test of the tile then reads
// its leaf record and edge list from shared memory.  A tile whose slices do
// not fit the buffers, a tile holding points pass 1 did not locate, and every
// tile of a queue left in pass-1 order (below PART_MIN_QUEUE entries) read
// the index from global memory as k_leaf_t1 does.  Every wait is bounded: a
// wait that runs out makes the block stop staging (its later tiles read
// global memory, so the late copy is never read), is counted once in
// g_tma_timeouts, and before exiting the block waits (bounded again) for
// that copy.  Both slices start on 16-byte boundaries (pool allocations are
// 256-byte aligned; leaf records are 32 bytes, edge records 16) and their
// sizes are multiples of 16 bytes.  Measured on 2e7 C2 points (9.1M queued):
// 337 us against 283 us for k_leaf_t1 on the same leaf-ordered queue, whose
// per-warp gathers leaf order already makes one request per warp and leaf;
// the staging adds a block barrier and a wait per tile and copies every
// leaf of the tile's range.  It is therefore an option (pass-2 order 3).
constexpr int T1S_LEAVES = 256;  // 8 KB of leaf records per tile
constexpr int T1S_RECS = 1536;   // 24 KB of edge records per tile
constexpr int T1S_BLOCKS = 5;

__global__ void __launch_bounds__(TPB, T1S_BLOCKS) k_leaf_t1s(QueryView Q, const double2* __restrict__ ll,
                                                            uint8_t* __restrict__ out,
                                                            const uint32_t* __restrict__ queue,
                                                            const unsigned int* __restrict__ qcount, Tiers T,
                                                            unsigned long long* ctr, int polls)
{
    __shared__ __align__(16) LeafRec s_leaf[T1S_LEAVES];
    __shared__ __align__(16) float4 s_rec[T1S_RECS];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ unsigned int s_wcnt[TPB / 32];
    __shared__ unsigned int s_base;
    __shared__ uint32_t s_l0, s_r0, s_nr;  // first staged leaf, first staged record, records staged
    __shared__ int s_nl;                   // leaves staged for the tile (0: none)
    __shared__ int s_broken;               // a wait ran out: no more staging
    if (threadIdx.x == 0) {
        mbar_init(&s_bar);
        s_broken = 0;
    }
    __syncthreads();
    wait_for_predecessor();
    const unsigned int m = *qcount;
    const uint32_t* src = queue;
    const uint32_t* src_leaf = T.l1;
    unsigned int st;
    first_tier_source(T, src, src_leaf, st);
    const bool sorted = src_leaf != T.l1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inside = 0, boundary = 0, fp64 = 0;
    uint32_t phase = 0;  // parity of the barrier's current phase
    // Thread 0 works a tile ahead so that a tile's copy goes out as the tile
    // starts: while the block labels tile k it loads the first and last leaf
    // words of tile k + 1, and after the labels those leaves' record
    // offsets (the bounds, state 1; 2 when the slices do not fit).
    // (thread 0's state is kept in shared memory, off the other threads'
    // registers)
    const unsigned int bstep = gridDim.x * blockDim.x;
    __shared__ uint32_t s_nw0, s_nw1;                 // next tile's first and last leaf words
    __shared__ uint32_t s_bL0, s_bL1, s_br0, s_br1;  // its leaves and record range
    __shared__ int s_bstate;                          // 0 not known, 1 staged, 2 not staged
    auto tile_words = [&](unsigned int b) {
        s_nw0 = src_leaf[b * st];
        s_nw1 = src_leaf[(min(b + TPB, m) - 1) * st];
    };
    auto tile_bounds = [&]() {
        const uint32_t w0 = s_nw0, w1 = s_nw1;
        s_bstate = 2;
        if ((w0 & KIND_MASK) != KIND_LEAF || (w1 & KIND_MASK) != KIND_LEAF) return;
        const uint32_t L0 = w0 & INDEX_MASK, L1 = w1 & INDEX_MASK;
        if (L1 < L0 || L1 - L0 >= (uint32_t)T1S_LEAVES) return;
        const uint32_t r0 = Q.leaves[L0].off, r1 = Q.leaves[L1].off + Q.leaves[L1].cnt;
        if (r1 < r0 || r1 - r0 > (uint32_t)T1S_RECS) return;
        s_bL0 = L0;
        s_bL1 = L1;
        s_br0 = r0;
        s_br1 = r1;
        s_bstate = 1;
    };
    if (threadIdx.x == 0) s_bstate = 0;
    if (threadIdx.x == 0 && sorted && blockIdx.x * blockDim.x < m) tile_words(blockIdx.x * blockDim.x);
    for (unsigned int b0 = blockIdx.x * blockDim.x; b0 < m; b0 += bstep) {
        if (threadIdx.x == 0) {
            int nl = 0;
            if (sorted && !s_broken) {
                if (s_bstate == 0) tile_bounds();  // the first tile
                if (s_bstate == 1) {
                    const uint32_t bL0 = s_bL0, br0 = s_br0;
                    nl = (int)(s_bL1 - bL0 + 1);
                    s_l0 = bL0;
                    s_r0 = br0;
                    s_nr = s_br1 - br0;
                    const uint32_t lb = (uint32_t)nl * (uint32_t)sizeof(LeafRec);
                    const uint32_t rb = (s_br1 - br0) * (uint32_t)sizeof(float4);
                    // the previous tile's reads of the buffers (ordered by
                    // the block barrier) come before these writes
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&s_bar)),
                                 "r"(lb + rb)
                                 : "memory");
                    asm volatile(
                        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                            smem_u32(s_leaf)),
                        "l"(Q.leaves + bL0), "r"(lb), "r"(smem_u32(&s_bar))
                        : "memory");
                    if (rb)
                        asm volatile(
                            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
                            "[%3];" ::"r"(smem_u32(s_rec)),
                            "l"(Q.recs + br0), "r"(rb), "r"(smem_u32(&s_bar))
                            : "memory");
                }
            }
            s_nl = nl;
            s_bstate = 0;
            if (sorted && b0 + bstep < m) tile_words(b0 + bstep);
        }
        // every thread's point and frame while the copy is in flight
        const unsigned int t = b0 + threadIdx.x;
        bool defer = false;
        uint32_t i = 0, w = 0, mask = 0;
        PointCtx P;
        if (t < m) {
            i = src[t * st];
            w = point_leaf(Q, ll[i], P, src_leaf[t * st]);
        }
        __syncthreads();
        const int nl = s_nl;
        bool staged = false;
        if (nl) {
            staged = mbar_wait(&s_bar, phase, polls);
            phase ^= 1u;
            if (!staged) atomicOr(&s_broken, 1);  // any thread whose wait ran out
        }
        if (t < m) {
            uint8_t lab;
            if ((w & KIND_MASK) == KIND_PURE) {
                lab = (uint8_t)(w & 3u);
            } else {
                boundary++;
                const uint32_t li = (w & INDEX_MASK) - s_l0;  // wraps above nl below the first leaf
                bool done = false;
                if (staged && li < (uint32_t)nl) {
                    const LeafRec L = s_leaf[li];
                    const uint32_t ro = L.off - s_r0;
                    if (ro <= s_nr && (uint32_t)L.cnt <= s_nr - ro) {
                        lab = leaf_label_fp32_at<true>(s_rec + ro, L, P, mask);
                        done = true;
                    }
                }
                if (!done) lab = leaf_label_fp32(Q, Q.leaves[w & INDEX_MASK], P, mask);
            }
            if (lab == LABEL_DEFER) {
                fp64++;
                defer = true;
            } else {
                out[i] = lab;
                inside += lab == CELL_IN;
            }
        }
        if (threadIdx.x == 0 && sorted && b0 + bstep < m) tile_bounds();  // the next tile's, ahead of its start
        const unsigned int bal = __ballot_sync(0xffffffffu, defer);
        if (lane == 0) s_wcnt[warp] = __popc(bal);
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned int tot = 0;
            for (int k = 0; k < TPB / 32; k++) {
                const unsigned int c = s_wcnt[k];
                s_wcnt[k] = tot;
                tot += c;
            }
            s_base = tot ? atomicAdd(T.cnt, tot) : 0u;
        }
        __syncthreads();
        if (defer) {
            const unsigned int pos = s_base + s_wcnt[warp] + __popc(bal & ((1u << lane) - 1u));
            if (pos < T.cap2) {
                T.q2[pos] = i;
                T.l2[pos] = w;
                T.m2[pos] = mask;
            } else {
                T.cnt[2] = 1;  // the tier-3 sweep labels it
            }
        }
        __syncthreads();  // s_wcnt / s_base and the staged slices are rewritten next round
    }
    allow_dependents();
    if (threadIdx.x == 0 && s_broken) {
        atomicAdd(&g_tma_timeouts, 1u);
        mbar_wait(&s_bar, phase ^ 1u);  // the copy whose wait ran out
    }
    if (ctr) count_stats(ctr, inside, boundary, fp64, 0);
}

// Tier 2's shape: blocks of 128 threads, five per SM (96 registers, about
// 60 bytes spilled) hold 20 warps per SM where 256-thread blocks at 110
// registers held 16: FP64-filter queries of C2 (tier 2 over the whole
// pass-1 queue) 15.8 -> 16.6 Gpts/s; six blocks (80 registers, 200 bytes
// spilled) 12.8; the FP32 filter's tier 2 is unchanged by any of them.
constexpr int T2_TPB = 128;
constexpr int T2_BLOCKS = 5;

// Tier 2 over the tier-1 queue, or (FROM_PASS1, FP64-filter queries) over
// the pass-1 queue itself.
template <class VS, bool FROM_PASS1>
__global__ void __launch_bounds__(T2_TPB, T2_BLOCKS) k_leaf_t2(VS vs, const double2* __restrict__ ll, uint8_t* __restrict__ out,
                                                const uint32_t* __restrict__ src, const uint32_t* __restrict__ src_leaf,
                                                const unsigned int* __restrict__ src_count, unsigned int src_cap,
                                                Tiers T, unsigned long long* ctr)
{
    wait_for_predecessor();
    const unsigned int m = min(*src_count, src_cap);
    const uint32_t* sp = src;
    const uint32_t* sl = src_leaf;
    unsigned int st = 1;
    if (FROM_PASS1) first_tier_source(T, sp, sl, st);
    int inside = 0, boundary = 0, exact = 0;
    for (unsigned int t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
        const uint32_t i = sp[t * st];
        const QueryView& Q = vs.of(i);
        PointCtx P;
        const uint32_t w = point_leaf(Q, ll[i], P, sl[t * st]);
        uint8_t lab;
        if ((w & KIND_MASK) == KIND_PURE) {
            lab = (uint8_t)(w & 3u);
        } else {
            if (FROM_PASS1) boundary++;
            lab = leaf_label_fp64(Q, w & INDEX_MASK, P, FROM_PASS1 ? MASK_ALL : T.m2[t]);
            if (lab == LABEL_DEFER) {
                exact++;
                if (!push_deferred(i, w, T.q3, T.l3, T.cnt + 1, T.cap3)) T.cnt[2] = 1;
                continue;
            }
        }
        out[i] = lab;
        inside += lab == CELL_IN;
    }
    allow_dependents();
    if (ctr) count_stats(ctr, inside, boundary, 0, exact);
}

// Tier 3 over the tier-2 queue, then, after a queue overflow, the complete
// test for every pass-1 point still unlabelled.
template <class VS>
__global__ void __launch_bounds__(TPB) k_leaf_t3(VS vs, const double2* __restrict__ ll, uint8_t* __restrict__ out,
                                                const uint32_t* __restrict__ queue,
                                                const unsigned int* __restrict__ qcount, Tiers T,
                                                unsigned long long* ctr)
{
    wait_for_predecessor();
    const unsigned int m3 = min(T.cnt[1], T.cap3);
    const bool sweep = T.cnt[2] != 0;
    const unsigned int m = sweep ? *qcount : 0;
    int inside = 0;
    for (unsigned int t = blockIdx.x * blockDim.x + threadIdx.x; t < m3 + m; t += gridDim.x * blockDim.x) {
        uint32_t i, known;
        if (t < m3) {
            i = T.q3[t];
            known = T.l3[t];
        } else {
            i = queue[t - m3];
            if (out[i] != LABEL_PENDING) continue;
            known = T.l1[t - m3];
        }
        const QueryView& Q = vs.of(i);
        PointCtx P;
        const uint32_t w = point_leaf(Q, ll[i], P, known);
        const uint8_t lab = ((w & KIND_MASK) == KIND_PURE) ? (uint8_t)(w & 3u)
                                                            : leaf_label(Q, w & INDEX_MASK, P, false, nullptr);
        out[i] = lab;
        inside += lab == CELL_IN;
    }
    if (ctr) count_inside(inside, ctr + 3);
}

// ------------------------------------- pass-2 queue in leaf-window order --
//
// Pass 1 queues points in input order, so on inputs without spatial order
// (C2's near-edge points) the tiers' gathers of leaf and edge records sweep
// the whole index, which is larger than L2 (350-400 MB on the C1 polygon):
// nearly every record comes from DRAM, once per point.  Leaves are numbered
// so that their records are contiguous, so a window of consecutive leaves is
// a contiguous slice of the index.  Two launches put the queue in window
// order (a counting sort with a few dozen bins, block-aggregated):
//   k_part_count    entries per window (shared-memory counts, one global
//                   atomic per window and block);
//   k_part_scatter  each block ranks a tile's entries per window in shared
//                   memory, takes the tile's place in each window with one
//                   global atomic per window, and writes them there.
// The tiers' grid-stride loops then sweep the queue in order, so at any time
// the grid works in one or two windows whose records stay in L2, and tier 1
// writes the tier-2 queue in the same order.  Windows are sized at about
// PART_BYTES of index; queues below PART_MIN_QUEUE entries keep pass-1 order
// (both kernels return at once and the tiers read the pass-1 queue).
constexpr int PART_MAX = 64;
constexpr long long PART_BYTES = 24LL << 20;
constexpr unsigned int PART_MIN_QUEUE = 1u << 18;
constexpr int P_TPB = 256;
constexpr int P_ITEMS = 8;

struct PartScratch {
    unsigned int* total;   // [PART_MAX] entries per window; zero before the pass
    unsigned int* cursor;  // [PART_MAX] entries placed per window; zero before the pass
    unsigned int* done;    // set to 1 when the window-ordered arrays are complete; zero before the pass
    uint32_t* spts;        // point indices in window order
    uint32_t* sleaf;       // their leaf words
    int np;                // windows (>= 2)
    float scale;           // QueryView::part_scale
};

__device__ __forceinline__ int part_of(uint32_t w, int np, float scale)
{
    if ((w & KIND_MASK) != KIND_LEAF) return np - 1;  // a point pass 1 did not locate
    return min((int)(__uint2float_rz(w & INDEX_MASK) * scale), np - 1);
}

// Adds one per active lane to cnt[b] in shared memory, one atomic per group
// of lanes with the same b; returns the lane's rank (old value + position).
__device__ __forceinline__ unsigned int smem_rank(unsigned int* cnt, int b)
{
    const unsigned int act = __activemask();
    const unsigned int same = __match_any_sync(act, b);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(same) - 1;
    unsigned int base = 0;
    if (lane == leader) base = atomicAdd(cnt + b, (unsigned int)__popc(same));
    base = __shfl_sync(same, base, leader);
    return base + __popc(same & ((1u << lane) - 1u));
}

__global__ void __launch_bounds__(P_TPB) k_part_count(const uint32_t* __restrict__ l1,
                                                      const unsigned int* __restrict__ qcount, PartScratch S)
{
    __shared__ unsigned int s_cnt[PART_MAX];
    wait_for_predecessor();
    const unsigned int m = *qcount;
    if (m < PART_MIN_QUEUE) {
        allow_dependents();
        return;
    }
    for (int k = threadIdx.x; k < S.np; k += P_TPB) s_cnt[k] = 0;
    __syncthreads();
    for (unsigned int t = blockIdx.x * P_TPB + threadIdx.x; t < m; t += gridDim.x * P_TPB)
        smem_rank(s_cnt, part_of(l1[t], S.np, S.scale));
    __syncthreads();
    allow_dependents();
    for (int k = threadIdx.x; k < S.np; k += P_TPB)
        if (s_cnt[k]) atomicAdd(S.total + k, s_cnt[k]);
}

__global__ void __launch_bounds__(P_TPB) k_part_scatter(const uint32_t* __restrict__ queue,
                                                        const uint32_t* __restrict__ l1,
                                                        const unsigned int* __restrict__ qcount, PartScratch S)
{
    __shared__ unsigned int s_start[PART_MAX], s_cnt[PART_MAX], s_base[PART_MAX];
    wait_for_predecessor();
    const unsigned int m = *qcount;
    if (m < PART_MIN_QUEUE) {
        allow_dependents();
        return;
    }
    if (threadIdx.x == 0) {
        unsigned int run = 0;
        for (int k = 0; k < S.np; k++) {
            s_start[k] = run;
            run += S.total[k];
        }
    }
    for (int k = threadIdx.x; k < S.np; k += P_TPB) s_cnt[k] = 0;
    __syncthreads();
    constexpr int TILE = P_TPB * P_ITEMS;
    // block-uniform loop; per tile: ranks (s_cnt), barrier, the tile's place
    // in each window (s_base; s_cnt cleared), barrier, writes
    for (unsigned int base = blockIdx.x * TILE; base < m; base += gridDim.x * TILE) {
        uint32_t q[P_ITEMS], w[P_ITEMS];
        unsigned int r[P_ITEMS];
        int b[P_ITEMS];
#pragma unroll
        for (int k = 0; k < P_ITEMS; k++) {
            const unsigned int t = base + k * P_TPB + threadIdx.x;
            q[k] = t < m ? queue[t] : 0u;
            w[k] = t < m ? l1[t] : 0u;
            b[k] = part_of(w[k], S.np, S.scale);
        }
#pragma unroll
        for (int k = 0; k < P_ITEMS; k++)
            if (base + k * P_TPB + threadIdx.x < m) r[k] = smem_rank(s_cnt, b[k]);
        __syncthreads();
        for (int j = threadIdx.x; j < S.np; j += P_TPB) {
            const unsigned int c = s_cnt[j];
            if (c) s_base[j] = s_start[j] + atomicAdd(S.cursor + j, c);
            s_cnt[j] = 0;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < P_ITEMS; k++) {
            if (base + k * P_TPB + threadIdx.x >= m) continue;
            const unsigned int at = s_base[b[k]] + r[k];
            if (at < m) {  // counts and entries agree; never write past the queue
                S.spts[at] = q[k];
                S.sleaf[at] = w[k];
            }
        }
    }
    allow_dependents();
    if (blockIdx.x == 0 && threadIdx.x == 0) *S.done = 1u;
}

// --------------------------------------- pass-2 queue in leaf order --
//
// The finest order: a counting sort of the pass-1 queue by leaf, so that the
// points of one leaf sit together and the warps of the first tier mostly
// take points of one leaf (their loads of the leaf's record and edge records
// are then one request per warp, served by L1 after the first).  Four
// launches:
//   k_ls_count      each entry takes its rank in its leaf (an atomic on the
//                   leaf's count; the last bucket holds points pass 1 did not
//                   locate);
//   k_ls_tile_sums  the counts' sums per tile of LS_TILE leaves;
//   k_ls_scan       each block scans one tile, starting from the sum of the
//                   tiles before it (no waits between blocks);
//   k_ls_scatter    each entry goes to its leaf's start plus its rank, point
//                   index and leaf word as one 8-byte pair (one random store
//                   per entry, where two arrays took two).
// The counts, ranks and the sorted arrays of a C2 pass fit in L2, so the
// random atomics and writes of the sort do not reach DRAM.
constexpr int LS_TPB = 256;
constexpr int LS_ITEMS = 16;
constexpr int LS_TILE = LS_TPB * LS_ITEMS;

struct LeafSortScratch {
    unsigned int* cnt;    // [nb] entries per bucket; zero before the pass
    unsigned int* start;  // [nb + 1] exclusive prefix of cnt
    unsigned int* tsum;   // [tiles] sums of cnt per tile
    unsigned int* rank;   // [queue] an entry's rank in its bucket
    uint2* sent;          // (point index, leaf word) in leaf order: one 8-byte store per entry
    unsigned int* done;   // set to 1 with the sorted arrays; zero before the pass
    int nb;               // buckets: leaves + 1
    int tiles;            // ceil(nb / LS_TILE)
    bool stage;           // tier 1 stages each tile's edge lists (k_leaf_t1s)
};

__device__ __forceinline__ int leaf_bucket(uint32_t w, int nb)
{
    return (w & KIND_MASK) == KIND_LEAF ? (int)min(w & INDEX_MASK, (uint32_t)(nb - 1)) : nb - 1;
}

__global__ void __launch_bounds__(LS_TPB) k_ls_count(const uint32_t* __restrict__ l1,
                                                     const unsigned int* __restrict__ qcount, LeafSortScratch S)
{
    wait_for_predecessor();
    const unsigned int m = *qcount;
    if (m >= PART_MIN_QUEUE)
        for (unsigned int t = blockIdx.x * LS_TPB + threadIdx.x; t < m; t += gridDim.x * LS_TPB)
            S.rank[t] = atomicAdd(S.cnt + leaf_bucket(l1[t], S.nb), 1u);
    allow_dependents();
}

// Block-wide sum of one value per thread (every thread gets it).
__device__ __forceinline__ unsigned int ls_block_sum(unsigned int v, unsigned int* s_w)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();  // s_w may still be read from the previous call
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = v;
    __syncthreads();
    unsigned int t = 0;
#pragma unroll
    for (int k = 0; k < LS_TPB / 32; k++) t += s_w[k];
    return t;
}

__global__ void __launch_bounds__(LS_TPB) k_ls_tile_sums(const unsigned int* __restrict__ qcount, LeafSortScratch S)
{
    __shared__ unsigned int s_w[LS_TPB / 32];
    wait_for_predecessor();
    if (*qcount >= PART_MIN_QUEUE) {
        for (int tile = blockIdx.x; tile < S.tiles; tile += gridDim.x) {
            unsigned int v = 0;
            const int b0 = tile * LS_TILE;
            for (int k = threadIdx.x; k < LS_TILE; k += LS_TPB)
                if (b0 + k < S.nb) v += S.cnt[b0 + k];
            v = ls_block_sum(v, s_w);
            if (threadIdx.x == 0) S.tsum[tile] = v;
        }
    }
    allow_dependents();
}

__global__ void __launch_bounds__(LS_TPB) k_ls_scan(const unsigned int* __restrict__ qcount, LeafSortScratch S)
{
    __shared__ unsigned int s_w[LS_TPB / 32];
    __shared__ unsigned int s_wx[LS_TPB / 32];
    wait_for_predecessor();
    if (*qcount >= PART_MIN_QUEUE) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int tile = blockIdx.x; tile < S.tiles; tile += gridDim.x) {
            unsigned int before = 0;
            for (int k = threadIdx.x; k < tile; k += LS_TPB) before += S.tsum[k];
            before = ls_block_sum(before, s_w);
            // this thread's LS_ITEMS consecutive buckets
            const int b0 = tile * LS_TILE + threadIdx.x * LS_ITEMS;
            unsigned int c[LS_ITEMS], run = 0;
#pragma unroll
            for (int k = 0; k < LS_ITEMS; k++) {
                c[k] = b0 + k < S.nb ? S.cnt[b0 + k] : 0u;
                run += c[k];
            }
            // exclusive scan of the threads' totals: in the warp, then over warps
            unsigned int x = run;
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            __syncthreads();  // s_wx may still be read from the previous tile
            if (lane == 31) s_wx[warp] = x;
            __syncthreads();
            unsigned int wbase = 0;
            for (int k = 0; k < warp; k++) wbase += s_wx[k];
            unsigned int at = before + wbase + x - run;
#pragma unroll
            for (int k = 0; k < LS_ITEMS; k++) {
                if (b0 + k < S.nb) S.start[b0 + k] = at;
                at += c[k];
            }
            if (b0 <= S.nb - 1 && S.nb - 1 < b0 + LS_ITEMS) S.start[S.nb] = at;  // the total
        }
    }
    allow_dependents();
}

__global__ void __launch_bounds__(LS_TPB) k_ls_scatter(const uint32_t* __restrict__ queue,
                                                       const uint32_t* __restrict__ l1,
                                                       const unsigned int* __restrict__ qcount, LeafSortScratch S)
{
    wait_for_predecessor();
    const unsigned int m = *qcount;
    if (m >= PART_MIN_QUEUE) {
        for (unsigned int t = blockIdx.x * LS_TPB + threadIdx.x; t < m; t += gridDim.x * LS_TPB) {
            const uint32_t w = l1[t];
            const unsigned int at = S.start[leaf_bucket(w, S.nb)] + S.rank[t];
            if (at < m) {  // counts and entries agree; never write past the queue
                S.sent[at] = make_uint2(queue[t], w);
            }
        }
    }
    allow_dependents();
    if (m >= PART_MIN_QUEUE && blockIdx.x == 0 && threadIdx.x == 0) *S.done = 1u;
}

// Launch with programmatic stream serialization (see wait_for_predecessor).
template <typename... KArgs, typename... Args>
void launch_dependent_tpb(void (*kernel)(KArgs...), int grid, int tpb, cudaStream_t s, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(tpb);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <typename... KArgs, typename... Args>
void launch_dependent(void (*kernel)(KArgs...), int grid, cudaStream_t s, Args... args)
{
    launch_dependent_tpb(kernel, grid, TPB, s, args...);
}

// Tier counters (T.cnt[0..2]) must be zero.  stage_t1 (one polygon, queue
// in leaf order): tier 1 reads each tile's edge lists from shared memory
// (k_leaf_t1s).
template <class VS>
void leaf_tiers_launch(const VS& vs, const double2* ll, uint8_t* out, const uint32_t* queue,
                       const unsigned int* qcount, const Tiers& T, int precision, unsigned long long* ctr, int sms,
                       cudaStream_t s, bool stage_t1 = false)
{
    if (precision == GAHHG_QUERY_FP64_FILTER) {
        launch_dependent_tpb(k_leaf_t2<VS, true>, sms * T2_BLOCKS, T2_TPB, s, vs, ll, out, queue,
                             (const uint32_t*)T.l1, qcount, 0xffffffffu, T, ctr);
    } else {
        bool staged = false;
        if constexpr (std::is_same<VS, OneView>::value) {
            if (stage_t1) {
                launch_dependent(k_leaf_t1s, sms * T1S_BLOCKS, s, vs.Q, ll, out, queue, qcount, T, ctr,
                                 (int)knob(GAHHG_KNOB_STAGING_POLL_LIMIT));
                staged = true;
            }
        }
        if (!staged) launch_dependent(k_leaf_t1<VS>, sms * T1_BLOCKS, s, vs, ll, out, queue, qcount, T, ctr);
        launch_dependent_tpb(k_leaf_t2<VS, false>, sms * T2_BLOCKS, T2_TPB, s, vs, ll, out, (const uint32_t*)T.q2,
                             (const uint32_t*)T.l2, (const unsigned int*)T.cnt, T.cap2, T, ctr);
    }
    launch_dependent(k_leaf_t3<VS>, sms * 2, s, vs, ll, out, queue, qcount, T, ctr);
}

// Escalation queue capacities for a pass-2 queue of `points` entries.
inline void tier_caps(long long points, unsigned int* cap2, unsigned int* cap3)
{
    *cap2 = (unsigned int)(points / 2 + 1024);
    *cap3 = (unsigned int)(points / 8 + 1024);
}

}  // namespace

// ------------------------------------------------------------------ host --

struct Lattice {
    Geo geo{};
    int K = 8, maxlev = 10, nlev = 0;
    DevArray<uint32_t> nodes;
    DevArray<LeafRec> leaves;
    DevArray<float4> recs;
    DevArray<uint32_t> eids;
    DevArray<double2> ends;
    DevArray<double> leafR;
    DevArray<uint32_t> summary;
    int cshift = 0, swords = 0;
    long long nedges = 0;
    int outside_label = 0;
    long long nnodes = 0, nleaves = 0, nrecs = 0;
    int origin_label = 0;
    double x_in[3]{};
};

void lattice_free(Lattice* L)
{
    if (!L) return;
    L->nodes.release();
    L->leaves.release();
    L->recs.release();
    L->eids.release();
    L->ends.release();
    L->leafR.release();
    L->summary.release();
    delete L;
}

size_t lattice_bytes(const Lattice* L)
{
    if (!L) return 0;
    return L->nnodes * sizeof(uint32_t) + L->nleaves * (sizeof(LeafRec) + 3 * sizeof(double)) +
           L->nrecs * (sizeof(float4) + sizeof(uint32_t)) + L->nedges * 3 * sizeof(double2);
}

size_t lattice_device_bytes(const Lattice* L)
{
    if (!L) return 0;
    return L->nodes.cap * sizeof(uint32_t) + L->leaves.cap * sizeof(LeafRec) + L->recs.cap * sizeof(float4) +
           L->eids.cap * sizeof(uint32_t) + L->ends.cap * sizeof(double2) + L->summary.cap * sizeof(uint32_t) +
           L->leafR.cap * sizeof(double);
}

namespace {

struct LevelBuf {
    int nn = 0;     // nodes at this level
    int gstart = 0; // global index of the first node
    DevArray<int> cnt, off, cursor, list, pair_node, child_base, flag, foff;
    DevArray<long long> ix, iy;
    DevArray<uint8_t> label;
    DevArray<int> poly;  // group builds: each node's polygon
    int npairs = 0;
    void release()
    {
        poly.release();
        cnt.release();
        off.release();
        cursor.release();
        list.release();
        pair_node.release();
        child_base.release();
        flag.release();
        foff.release();
        ix.release();
        iy.release();
        label.release();
    }
};

// Sorts every cell list: short ones by their own thread, long ones by a whole
// block each (k_sort_long), so no thread holds its block for long.
gahhg_status sort_lists(Grid* g, const int* cnt, const int* off, int nn, int* list, int sms, cudaStream_t s)
{
    int* d_nlong = g->d_counts + 20;  // [0] long lists, [1] next list to sort
    GAHHG_CUDA_TRY(cudaMemsetAsync(d_nlong, 0, 2 * sizeof(int), s));
    DevArray<int> long_ids;
    GAHHG_TRY(long_ids.reserve(std::max(nn, 1), s, false));
    k_sort_lists<<<blocks_for(nn), TPB, 0, s>>>(cnt, off, nn, list, long_ids.ptr, d_nlong);
    k_sort_long<<<sms * 2, SORT_TPB, 0, s>>>(cnt, off, list, long_ids.ptr, d_nlong, d_nlong + 1);
    GAHHG_CUDA_TRY(cudaGetLastError());
    return GAHHG_OK;
}

const double HUBS[6][3] = {
    {1.0, 0.000731, 0.000419},  {-1.0, 0.000627, -0.000883}, {0.000577, 1.0, 0.000941},
    {-0.000351, -1.0, 0.000713}, {0.000809, -0.000467, 1.0}, {-0.000689, 0.000523, -1.0},
};

// parity of all edges crossing arc P->Q (device), -1 on vertex coincidence
gahhg_status arc_parity_all(Grid* g, const double* P, const double* Q, int* parity, int* ncross, int* last_edge)
{
    cudaStream_t s = g->stream;
    double* d_pq = reinterpret_cast<double*>(g->d_counts + 40);  // 6 doubles in the counts scratch (8-aligned)
    double pq[6] = {P[0], P[1], P[2], Q[0], Q[1], Q[2]};
    int* d_out = g->d_counts + 56;
    GAHHG_CUDA_TRY(cudaMemcpyAsync(d_pq, pq, sizeof(pq), cudaMemcpyHostToDevice, s));
    int init[4] = {0, 0, 0, -1};
    GAHHG_CUDA_TRY(cudaMemcpyAsync(d_out, init, sizeof(init), cudaMemcpyHostToDevice, s));
    const int n = g->poly->pv_num;
    k_arc_parity_all<<<blocks_for(n), TPB, 0, s>>>(g->poly->d_pv, g->poly->d_pe, n, d_pq, d_out);
    int out[4];
    GAHHG_CUDA_TRY(cudaMemcpyAsync(out, d_out, sizeof(out), cudaMemcpyDeviceToHost, s));
    GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
    *parity = out[1] ? -1 : out[0];
    if (ncross) *ncross = out[2];
    if (last_edge) *last_edge = out[3];
    return GAHHG_OK;
}

// A point just left of an outer-ring edge (the exact oracle takes the same
// steps: first usable edge, offset 1e-3 * chord along the edge normal, the
// tiny arc from its mirror image crossing exactly this one edge).
gahhg_status reference_point(Grid* g, double* x_in)
{
    const Polygon* P = g->poly;
    const int n_outer = P->ring_start[1];
    for (int e = 0; e < n_outer; e++) {
        const D3 a = P->pv[P->pe[2 * e]], b = P->pv[P->pe[2 * e + 1]];
        const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z};
        if (exact::same(A, B)) continue;
        double m[3] = {A[0] + B[0], A[1] + B[1], A[2] + B[2]};
        double nm = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
        if (!(nm > 1e-3)) continue;
        double N[3] = {A[1] * B[2] - A[2] * B[1], A[2] * B[0] - A[0] * B[2], A[0] * B[1] - A[1] * B[0]};
        double nn = sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
        if (!(nn > 0)) continue;
        double d[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
        double t = 1e-3 * sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        double xi[3], xo[3];
        for (int k = 0; k < 3; k++) {
            xi[k] = m[k] / nm + t * (N[k] / nn);
            xo[k] = m[k] / nm - t * (N[k] / nn);
        }
        if (exact::orient(A, B, xi) <= 0 || exact::orient(A, B, xo) >= 0) continue;
        int par, nc, le;
        GAHHG_TRY(arc_parity_all(g, xo, xi, &par, &nc, &le));
        if (par != 1 || nc != 1 || le != e) continue;
        memcpy(x_in, xi, sizeof(xi));
        return GAHHG_OK;
    }
    set_error("exact index: no outer-ring edge gives a reference point");
    return GAHHG_ERR_STATE;
}

int nearest_hub(const double* q)
{
    int best = 0;
    double bd = -1e300;
    for (int k = 0; k < 6; k++) {
        double d = HUBS[k][0] * q[0] + HUBS[k][1] * q[1] + HUBS[k][2] * q[2];
        if (d > bd) {
            bd = d;
            best = k;
        }
    }
    return best;
}

}  // namespace


// Longitude/latitude domain of the polygon's edges, padded by one cell, with
// cells of near-equal size in degrees whose count is about `target`.  A
// domain that reaches within a degree of a pole takes in the whole polar cap
// (all longitudes), so that points outside it are never close to an edge.
// Latitude range and touched 0.1-degree longitude bins of edges [e0, e1).
// The domain scan on the device: per edge its latitude range and the
// 0.1-degree longitude bins it touches (long edges by their great-circle box,
// short ones by their ends' latitude and longitude, padded by 1e-4 degrees),
// reduced per block in shared memory and then with one atomic per block and
// word.  Min, max and OR do not depend on the order of the edges.
constexpr int DOMAIN_BIN_WORDS = (3600 + 31) / 32;
struct DomainOut {
    unsigned long long latmin, latmax;  // order-preserving keys of the doubles
    unsigned int full;
    unsigned int bins[DOMAIN_BIN_WORDS];
};

__device__ __forceinline__ unsigned long long order_key(double x)
{
    const unsigned long long u = (unsigned long long)__double_as_longlong(x);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__host__ inline double from_order_key(unsigned long long k)
{
    const unsigned long long u = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
    double x;
    memcpy(&x, &u, sizeof x);
    return x;
}

__global__ void __launch_bounds__(TPB) k_domain_scan(const D3* __restrict__ pv, const int* __restrict__ pe, int n,
                                                     DomainOut* out)
{
    __shared__ unsigned int s_bins[DOMAIN_BIN_WORDS];
    __shared__ unsigned long long s_min, s_max;
    __shared__ unsigned int s_full;
    for (int k = threadIdx.x; k < DOMAIN_BIN_WORDS; k += TPB) s_bins[k] = 0;
    if (threadIdx.x == 0) {
        s_min = ~0ull;
        s_max = 0ull;
        s_full = 0;
    }
    __syncthreads();
    double lmin = 90.0, lmax = -90.0;
    bool full = false;
    for (int e = blockIdx.x * TPB + threadIdx.x; e < n; e += gridDim.x * TPB) {
        const D3 a = pv[pe[2 * e]], b = pv[pe[2 * e + 1]];
        if (a.x == b.x && a.y == b.y && a.z == b.z) continue;
        double la0, la1, lo0, lo1;
        bool fl = false;
        const double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
        if (dx * dx + dy * dy + dz * dz > 1e-4) {
            arc_box(a, b, la0, la1, lo0, lo1, fl);  // long edge: its great circle may bulge
        } else {
            // short edge: its ends (the bulge is below 1e-4 deg, far inside the one-cell padding)
            const double ta = lat_of(a), tb = lat_of(b);
            double oa = lon_of(a), ob = lon_of(b);
            la0 = fmin(ta, tb) - 1e-4;
            la1 = fmax(ta, tb) + 1e-4;
            if (oa > ob) {
                const double t = oa;
                oa = ob;
                ob = t;
            }
            if (ob - oa <= 180.0) {
                lo0 = oa;
                lo1 = ob;
            } else {
                lo0 = ob;
                lo1 = oa + 360.0;
            }
            if (fabs(ta) > 89.9 || fabs(tb) > 89.9) fl = true;
        }
        lmin = fmin(lmin, la0);
        lmax = fmax(lmax, la1);
        if (fl) {
            full = true;
            continue;
        }
        const int b0 = (int)floor((lo0 + 180.0) * 10.0) - 1, b1 = (int)floor((lo1 + 180.0) * 10.0) + 1;
        for (int k = b0; k <= b1 && k <= b0 + 3600; k++) {
            const int bit = ((k % 3600) + 3600) % 3600;
            atomicOr(&s_bins[bit >> 5], 1u << (bit & 31));
        }
    }
    for (int d = 16; d > 0; d >>= 1) {
        lmin = fmin(lmin, __shfl_down_sync(0xffffffffu, lmin, d));
        lmax = fmax(lmax, __shfl_down_sync(0xffffffffu, lmax, d));
    }
    full = __any_sync(0xffffffffu, full);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&s_min, order_key(lmin));
        atomicMax(&s_max, order_key(lmax));
        if (full) s_full = 1;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < DOMAIN_BIN_WORDS; k += TPB)
        if (s_bins[k]) atomicOr(&out->bins[k], s_bins[k]);
    if (threadIdx.x == 0) {
        atomicMin(&out->latmin, s_min);
        atomicMax(&out->latmax, s_max);
        if (s_full) atomicOr(&out->full, 1u);
    }
}

// ----------------------------------------------------------- group builds --
//
// A batch's polygons are built in groups: every step of the exact-index build
// runs once for all polygons of a group (shared launches over concatenated
// edges and nodes, a polygon table for the per-polygon geometry), so a
// group's launches and host round trips scale with its levels, not with its
// polygons.  The steps are those of lattice_build, node for node and edge for
// edge: a polygon's index is the one its own build gives, renumbered into the
// group's arrays (node words hold child indices relative to the polygon's
// first top node, so its query view sees its own numbering; leaves, records
// and edge ids are group-wide).


// base[0..n] ascending: the p with base[p] <= x < base[p + 1] (the last such
// p when ranges are empty)
__device__ __forceinline__ int find_range(const long long* __restrict__ base, int n, long long x)
{
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(base + mid) <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

// group edge -> polygon; the polygon's vertex indices shifted to the group's
__global__ void kb_edges(const long long* ebase, const long long* vbase, int np, long long ne, int* epoly, int* pe)
{
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= ne) return;
    const int p = find_range(ebase, np, e);
    epoly[e] = p;
    const int vb = (int)vbase[p];
    pe[2 * e] += vb;
    pe[2 * e + 1] += vb;
}

// k_domain_scan for every polygon of a group: per-edge results into the
// edge's polygon's DomainOut with global atomics (bins read first, so most
// edges set no bit that is already set)
__global__ void __launch_bounds__(TPB) kb_domain_scan(const D3* __restrict__ pv, const int* __restrict__ pe,
                                                      long long ne, const int* __restrict__ epoly, DomainOut* out)
{
    for (long long e0 = (long long)blockIdx.x * TPB; e0 < ne; e0 += (long long)gridDim.x * TPB) {
        const long long e = e0 + threadIdx.x;
        int p = -1;
        double la0 = 90.0, la1 = -90.0;
        bool fl = false, any = false;
        int b0 = 0, b1 = -1;
        if (e < ne) {
            p = epoly[e];
            const D3 a = pv[pe[2 * e]], b = pv[pe[2 * e + 1]];
            if (!(a.x == b.x && a.y == b.y && a.z == b.z)) {
                any = true;
                double lo0, lo1;
                const double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
                if (dx * dx + dy * dy + dz * dz > 1e-4) {
                    arc_box(a, b, la0, la1, lo0, lo1, fl);
                } else {
                    const double ta = lat_of(a), tb = lat_of(b);
                    double oa = lon_of(a), ob = lon_of(b);
                    la0 = fmin(ta, tb) - 1e-4;
                    la1 = fmax(ta, tb) + 1e-4;
                    if (oa > ob) {
                        const double t = oa;
                        oa = ob;
                        ob = t;
                    }
                    if (ob - oa <= 180.0) {
                        lo0 = oa;
                        lo1 = ob;
                    } else {
                        lo0 = ob;
                        lo1 = oa + 360.0;
                    }
                    if (fabs(ta) > 89.9 || fabs(tb) > 89.9) fl = true;
                }
                if (!fl) {
                    b0 = (int)floor((lo0 + 180.0) * 10.0) - 1;
                    b1 = (int)floor((lo1 + 180.0) * 10.0) + 1;
                }
            }
        }
        // a warp whose edges all belong to one polygon reduces before its atomics
        const unsigned int same = __match_any_sync(0xffffffffu, p);
        if (same == 0xffffffffu && p >= 0) {
            double mn = la0, mx = la1;
            for (int d = 16; d > 0; d >>= 1) {
                mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, d));
                mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, d));
            }
            const bool f = __any_sync(0xffffffffu, any && fl);
            const bool a = __any_sync(0xffffffffu, any);
            if ((threadIdx.x & 31) == 0 && a) {
                atomicMin(&out[p].latmin, order_key(mn));
                atomicMax(&out[p].latmax, order_key(mx));
                if (f) atomicOr(&out[p].full, 1u);
            }
        } else if (p >= 0 && any) {
            atomicMin(&out[p].latmin, order_key(la0));
            atomicMax(&out[p].latmax, order_key(la1));
            if (fl) atomicOr(&out[p].full, 1u);
        }
        if (p >= 0 && any && !fl) {
            for (int k = b0; k <= b1 && k <= b0 + 3600; k++) {
                const int bit = ((k % 3600) + 3600) % 3600;
                unsigned int* w = &out[p].bins[bit >> 5];
                if (!(*(volatile unsigned int*)w & (1u << (bit & 31)))) atomicOr(w, 1u << (bit & 31));
            }
        }
    }
}

// Parity, count and last index of the group edges [e0, e1) crossing arc
// P -> Q, summed over the block (as k_arc_parity_all); coincident is set
// when an edge end coincides with P or Q.  Every thread of the block calls.
__device__ void block_arc_parity(const D3* pv, const int* pe, long long e0, long long e1, const double* P,
                                 const double* Q, int& parity, int& ncross, int& last, bool& coincident)
{
    __shared__ int s_par, s_cnt, s_last, s_co;
    __syncthreads();
    if (threadIdx.x == 0) {
        s_par = 0;
        s_cnt = 0;
        s_last = -1;
        s_co = 0;
    }
    __syncthreads();
    int par = 0, cnt = 0, lst = -1, co = 0;
    for (long long e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const D3 a = pv[pe[2 * e]], b = pv[pe[2 * e + 1]];
        const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z};
        if (exact::same(A, B)) continue;
        if (exact::same(A, P) || exact::same(B, P) || exact::same(A, Q) || exact::same(B, Q)) {
            co = 1;
            continue;
        }
        if (exact::crossing(P, Q, A, B)) {
            par ^= 1;
            cnt++;
            lst = max(lst, (int)(e - e0));
        }
    }
    if (par) atomicXor(&s_par, 1);
    if (cnt) atomicAdd(&s_cnt, cnt);
    if (lst >= 0) atomicMax(&s_last, lst);
    if (co) s_co = 1;
    __syncthreads();
    parity = s_par;
    ncross = s_cnt;
    last = s_last;
    coincident = s_co != 0;
    __syncthreads();
}

__constant__ double c_hubs[6][3] = {
    {1.0, 0.000731, 0.000419},  {-1.0, 0.000627, -0.000883}, {0.000577, 1.0, 0.000941},
    {-0.000351, -1.0, 0.000713}, {0.000809, -0.000467, 1.0}, {-0.000689, 0.000523, -1.0},
};

__device__ int nearest_hub_d(const double* q)
{
    int best = 0;
    double bd = -1e300;
    for (int k = 0; k < 6; k++) {
        const double d = c_hubs[k][0] * q[0] + c_hubs[k][1] * q[1] + c_hubs[k][2] * q[2];
        if (d > bd) {
            bd = d;
            best = k;
        }
    }
    return best;
}

// One block per polygon: the reference point just left of an outer-ring
// edge (reference_point) and the exact label of the first level-0 center
// through the hubs (lattice_build's origin step).  origin[p] = the label, or
// 0 when no outer edge gives a reference point, -1 when a hub or the center
// coincides with a vertex.
constexpr int ORIGIN_TPB = 512;
__global__ void __launch_bounds__(ORIGIN_TPB) kb_origin(const D3* __restrict__ pv, const int* __restrict__ pe,
                                                 const PolyGeo* __restrict__ pg, const long long* __restrict__ ebase,
                                                 const int* __restrict__ nouter, int* origin)
{
    const int p = blockIdx.x;
    const long long e0 = ebase[p], e1 = ebase[p + 1];
    __shared__ double s_xi[3], s_xo[3];
    __shared__ int s_ok;
    bool found = false;
    double xin[3] = {0.0, 0.0, 0.0};
    for (int e = 0; e < nouter[p] && !found; e++) {
        __syncthreads();  // every thread has read the previous candidate's s_ok
        if (threadIdx.x == 0) {
            s_ok = 0;
            const D3 a = pv[pe[2 * (e0 + e)]], b = pv[pe[2 * (e0 + e) + 1]];
            const double A[3] = {a.x, a.y, a.z}, B[3] = {b.x, b.y, b.z};
            double m[3] = {A[0] + B[0], A[1] + B[1], A[2] + B[2]};
            const double nm = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
            const double N[3] = {A[1] * B[2] - A[2] * B[1], A[2] * B[0] - A[0] * B[2], A[0] * B[1] - A[1] * B[0]};
            const double nn = sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
            if (!exact::same(A, B) && nm > 1e-3 && nn > 0) {
                const double d[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
                const double t = 1e-3 * sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                double xi[3], xo[3];
                for (int k = 0; k < 3; k++) {
                    xi[k] = m[k] / nm + t * (N[k] / nn);
                    xo[k] = m[k] / nm - t * (N[k] / nn);
                }
                if (exact::orient(A, B, xi) > 0 && exact::orient(A, B, xo) < 0) {
                    for (int k = 0; k < 3; k++) {
                        s_xi[k] = xi[k];
                        s_xo[k] = xo[k];
                    }
                    s_ok = 1;
                }
            }
        }
        __syncthreads();
        if (!s_ok) continue;  // the same in every thread
        double xo[3] = {s_xo[0], s_xo[1], s_xo[2]}, xi[3] = {s_xi[0], s_xi[1], s_xi[2]};
        int par, nc, le;
        bool co;
        block_arc_parity(pv, pe, e0, e1, xo, xi, par, nc, le, co);
        if (!co && par == 1 && nc == 1 && le == e) {
            found = true;
            for (int k = 0; k < 3; k++) xin[k] = xi[k];
        }
    }
    if (!found) {
        if (threadIdx.x == 0) origin[p] = 0;
        return;
    }
    const NodeCap c00 = node_cap(pg[p].g, 0, 0, 0);
    double path[5][3];
    int np = 0;
    for (int k = 0; k < 3; k++) path[np][k] = xin[k];
    np++;
    const double ud = (xin[0] * c00.R[0] + xin[1] * c00.R[1] + xin[2] * c00.R[2]) /
                      sqrt((xin[0] * xin[0] + xin[1] * xin[1] + xin[2] * xin[2]) *
                           (c00.R[0] * c00.R[0] + c00.R[1] * c00.R[1] + c00.R[2] * c00.R[2]));
    if (ud < 0.1) {
        const int ha = nearest_hub_d(xin), hb = nearest_hub_d(c00.R);
        for (int k = 0; k < 3; k++) path[np][k] = c_hubs[ha][k];
        np++;
        if ((ha ^ 1) == hb) {
            for (int k = 0; k < 3; k++) path[np][k] = c_hubs[(ha + 2) % 6][k];
            np++;
        }
        if (hb != ha) {
            for (int k = 0; k < 3; k++) path[np][k] = c_hubs[hb][k];
            np++;
        }
    }
    for (int k = 0; k < 3; k++) path[np][k] = c00.R[k];
    np++;
    int label = CELL_IN;
    for (int k = 0; k + 1 < np; k++) {
        int par, nc, le;
        bool co;
        block_arc_parity(pv, pe, e0, e1, path[k], path[k + 1], par, nc, le, co);
        if (co) {
            if (threadIdx.x == 0) origin[p] = -1;
            return;
        }
        if (par) label = 3 - label;
    }
    if (threadIdx.x == 0) origin[p] = label;
}

// k_l0_box for the group's edges (each in its polygon's grid)
__global__ void kb_l0_box(const D3* __restrict__ pv, const int* __restrict__ pe, long long ne,
                          const int* __restrict__ epoly, const PolyGeo* __restrict__ pg, EdgeBox* box, int* items,
                          unsigned long long* total64)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long nit = 0;
    if (t < ne) {
        EdgeBox bx{0, 0, 0, 0, 0, 0};
        const D3 A = pv[pe[2 * t]], B = pv[pe[2 * t + 1]];
        if (!(A.x == B.x && A.y == B.y && A.z == B.z)) {
            const Geo& G = pg[epoly[t]].g;
            nit = edge_box(G, A, B, bx);
        }
        box[t] = bx;
        items[t] = (int)min(nit, (long long)INT_MAX);
    }
    unsigned long long w = (unsigned long long)nit;
    for (int d = 16; d > 0; d >>= 1) w += __shfl_down_sync(0xffffffffu, w, d);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd(total64, w);
}

// Level-0 node coordinates and polygons.
__global__ void kb_l0_coords(const long long* __restrict__ tops, int np, const PolyGeo* __restrict__ pg, int nn,
                             long long* ix, long long* iy, int* npoly)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nn) return;
    const int p = find_range(tops, np, v);
    const long long local = v - pg[p].top;
    const int W = pg[p].g.W;
    ix[v] = local % W;
    iy[v] = local / W;
    npoly[v] = p;
}

// k_l0_neighbour_parity for the group: per polygon its W (H - 1) vertical
// pairs, then its W - 1 horizontal pairs of row 0, from pb[p] in `par`.
__global__ void kb_l0_neighbour_parity(const D3* __restrict__ pv, const int* __restrict__ pe,
                                       const PolyGeo* __restrict__ pg, const long long* __restrict__ pb, int np,
                                       const int* cnt, const int* off, const int* list, uint8_t* par, int* bad)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= pb[np]) return;
    const int p = find_range(pb, np, t);
    const PolyGeo& P = pg[p];
    const int W = P.g.W, H = P.g.H;
    const long long u = t - pb[p];
    const long long nv = (long long)W * (H - 1);
    int i, j, i2, j2;
    if (u < nv) {
        i = (int)(u % W);
        j = (int)(u / W);
        i2 = i;
        j2 = j + 1;
    } else {
        i = (int)(u - nv);
        j = 0;
        i2 = i + 1;
        j2 = 0;
    }
    const long long a0 = P.top + (long long)j * W + i, b0 = P.top + (long long)j2 * W + i2;
    uint8_t r = 0;
    if (cnt[a0] || cnt[b0]) {
        NodeCap a = node_cap(P.g, 0, i, j), b = node_cap(P.g, 0, i2, j2);
        nudge_center(P.g, 0, a, pv, pe, list + off[a0], cnt[a0]);
        nudge_center(P.g, 0, b, pv, pe, list + off[b0], cnt[b0]);
        r = (uint8_t)arc_parity_lists(pv, pe, a.R, b.R, list + off[a0], cnt[a0], list + off[b0], cnt[b0], bad);
    }
    par[t] = r;
}

// k_l0_labels for the group: one thread per column of every polygon (cb[p]:
// the polygon's first column).
__global__ void kb_l0_labels(const PolyGeo* __restrict__ pg, const long long* __restrict__ cb,
                             const long long* __restrict__ pb, int np, const uint8_t* __restrict__ par,
                             const int* __restrict__ origin, uint8_t* label)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cb[np]) return;
    const int p = find_range(cb, np, t);
    const PolyGeo& P = pg[p];
    const int W = P.g.W, H = P.g.H;
    const int i = (int)(t - cb[p]);
    const uint8_t* vpar = par + pb[p];
    const uint8_t* hpar = vpar + (long long)W * (H - 1);
    int l = origin[p];  // 1 or 2
    for (int k = 0; k < i; k++)
        if (hpar[k]) l = 3 - l;
    label[P.top + i] = (uint8_t)l;
    for (int j = 1; j < H; j++) {
        if (vpar[(long long)(j - 1) * W + i]) l = 3 - l;
        label[P.top + (long long)j * W + i] = (uint8_t)l;
    }
}

// k_outside_label for every polygon with a region outside its domain
// (oxy[p] = (ix, iy, ox, oy) from the host, ox == INT_MIN: none).
__global__ void kb_outside_label(const D3* __restrict__ pv, const int* __restrict__ pe,
                                 const PolyGeo* __restrict__ pg, int np, const int4* __restrict__ oxy,
                                 const int* cnt, const int* off, const int* list, const uint8_t* label, uint8_t* out,
                                 int* bad)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const int4 o = oxy[p];
    if (o.z == INT_MIN) {
        out[p] = CELL_UNDEFINED;
        return;
    }
    const PolyGeo& P = pg[p];
    const long long v = P.top + (long long)o.y * P.g.W + o.x;
    NodeCap a = node_cap(P.g, 0, o.x, o.y);
    nudge_center(P.g, 0, a, pv, pe, list + off[v], cnt[v]);
    const NodeCap b = node_cap(P.g, 0, o.z, o.w);
    const int par = arc_parity_lists(pv, pe, a.R, b.R, list + off[v], cnt[v], nullptr, 0, bad);
    out[p] = (uint8_t)(par ? 3 - label[v] : label[v]);
}

__global__ void kb_refine_flags(const int* cnt, const int* npoly, const PolyGeo* __restrict__ pg, int nn, int* flag)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < nn) flag[v] = cnt[v] > pg[npoly[v]].K ? 1 : 0;
}

// k_make_children for the group: children take their parent's polygon
__global__ void kb_make_children(const int* flag, const int* foff, int nn, int cstart, const long long* pix,
                                 const long long* piy, const int* npoly, int* child_base, long long* cix,
                                 long long* ciy, int* cpoly)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nn) return;
    if (!flag[v]) {
        child_base[v] = -1;
        return;
    }
    child_base[v] = cstart + foff[v] * FAN * FAN;
    const long long px = pix[v], py = piy[v];
    for (int cy = 0; cy < FAN; cy++)
        for (int cx = 0; cx < FAN; cx++) {
            const int c = foff[v] * FAN * FAN + cy * FAN + cx;
            cix[c] = px * FAN + cx;
            ciy[c] = py * FAN + cy;
            cpoly[c] = npoly[v];
        }
}

__global__ void kb_child_caps(const PolyGeo* __restrict__ pg, int lvl, int nn, const long long* ix,
                              const long long* iy, const int* cpoly, double4* caps, double2* capsb)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nn) return;
    const NodeCap nc = node_cap(pg[cpoly[c]].g, lvl, ix[c], iy[c]);
    caps[c] = make_double4(nc.R[0], nc.R[1], nc.R[2], cap_chord2(nc.r));
    capsb[c] = make_double2(cap_sin_bound(nc.r), nc.r);
}

// k_summary for every polygon: coarse cell c of polygon p (sc[p]: its first
// cell in the group) into its summary words from soff[p]
__global__ void kb_summary(const uint32_t* nodes, const PolyGeo* __restrict__ pg, const long long* __restrict__ sc,
                           const int* __restrict__ cshift, const long long* __restrict__ soff, int np,
                           uint32_t* summary)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= sc[np]) return;
    const int p = find_range(sc, np, t);
    const int c = (int)(t - sc[p]);
    const int W = pg[p].g.W, H = pg[p].g.H, cs = cshift[p];
    const int f = 1 << cs;
    const int CW = (W + f - 1) >> cs;
    const int cx = c % CW, cy = c / CW;
    const uint32_t* top = nodes + pg[p].top;
    uint32_t code = 0xFFu;
    for (int y = cy * f; y < min((cy + 1) * f, H) && code != 2u; y++)
        for (int x = cx * f; x < min((cx + 1) * f, W); x++) {
            const uint32_t w = top[(size_t)y * W + x];
            const uint32_t v = ((w & KIND_MASK) == KIND_PURE) ? (w & 3u) - 1u : 2u;  // 0 out, 1 in, 2 mixed
            if (code == 0xFFu) code = v;
            else if (code != v) code = 2u;
            if (code == 2u) break;
        }
    atomicOr(&summary[soff[p] + (c >> 4)], code << ((c & 15) * 2));
}


gahhg_status geo_from_scan(const DomainOut& h, const Polygon* P, long long target, Geo* G);

gahhg_status compute_domain(const Polygon* P, long long target, Geo* G, cudaStream_t s, int device)
{
    DomainOut h;
    {
        DomainOut* d = nullptr;
        GAHHG_TRY(pool_alloc((void**)&d, sizeof(DomainOut), device, s));
        memset(&h, 0, sizeof h);
        h.latmin = ~0ull;
        GAHHG_CUDA_TRY(cudaMemcpyAsync(d, &h, sizeof h, cudaMemcpyHostToDevice, s));
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        const int grid = (int)std::max(1LL, std::min<long long>(sms * 4LL, (P->pv_num + TPB - 1) / TPB));
        k_domain_scan<<<grid, TPB, 0, s>>>(P->d_pv, P->d_pe, P->pv_num, d);
        GAHHG_CUDA_TRY(cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, s));
        cudaFreeAsync(d, s);
        GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
    }
    return geo_from_scan(h, P, target, G);
}

// The level-0 grid from the domain scan's result (host).
gahhg_status geo_from_scan(const DomainOut& h, const Polygon* P, long long target, Geo* G)
{
    double latmin = h.latmax == 0ull ? 90.0 : from_order_key(h.latmin);
    double latmax = h.latmax == 0ull ? -90.0 : from_order_key(h.latmax);
    bool full = h.full != 0;
    std::vector<uint8_t> bins(3600);  // 0.1-degree longitude bins touched by some arc
    for (int k = 0; k < 3600; k++) bins[k] = (h.bins[k >> 5] >> (k & 31)) & 1u;
    if (latmin > latmax) {
        set_error("exact index: polygon has no edges of positive length");
        return GAHHG_ERR_ARG;
    }
    // largest circular run of untouched bins = the longitude gap left outside
    int gstart = 0, glen = 0;
    if (!full) {
        int best = 0, bs = 0;
        for (int st = 0; st < 3600; st++) {
            if (bins[st] || bins[(st + 3599) % 3600] == 0) continue;  // runs start after a touched bin
            int len = 0;
            while (len < 3600 && !bins[(st + len) % 3600]) len++;
            if (len > best) {
                best = len;
                bs = st;
            }
        }
        gstart = bs;
        glen = best;
        if (glen == 0) full = true;
    }
    double lon0 = -180.0, lon_span = 360.0;
    if (!full) {
        lon0 = ((gstart + glen) % 3600) * 0.1 - 180.0;
        lon_span = (3600 - glen) * 0.1;
    }
    double lat_span = std::max(latmax - latmin, 1e-6);
    // Cells are `aspect` times wider in longitude than in latitude, so that
    // they are about square on the sphere at the median latitude of the
    // vertices; near a pole square-in-degrees cells are needles that every
    // edge crosses by the dozen.  Below an aspect of 2 cells stay square in
    // degrees.
    double aspect = 1.0;
    {
        // a strided sample of at most 65536 vertices is enough for the median
        const int stride = std::max(1, P->pv_num / 65536);
        std::vector<double> alat;
        alat.reserve(P->pv_num / stride + 1);
        for (int v = 0; v < P->pv_num; v += stride) alat.push_back(fabs(P->lonlat[2 * v + 1]));
        if (!alat.empty()) {
            std::nth_element(alat.begin(), alat.begin() + alat.size() / 2, alat.end());
            const double a = 1.0 / std::max(cos(std::min(alat[alat.size() / 2], 89.99) * RAD), 1e-9);
            if (a >= 2.0) aspect = std::min(a, 64.0);
        }
    }
    // cell height (degrees) for about `target` cells, with the padding included
    double cell = sqrt(std::max(lon_span, 1e-6) * lat_span / ((double)std::max(target, 1LL) * aspect));
    bool full_lon = full, north = false, south = false;
    for (int it = 0; it < 3; it++) {
        const double pad = cell * 1.5;
        double la = latmin - pad, lb = latmax + pad;
        north = lb >= 89.0;
        south = la <= -89.0;
        bool fl = full || north || south;
        double lspan = 360.0, l0 = -180.0;
        if (!fl) {
            const double maxabs = std::min(89.0, std::max(fabs(la), fabs(lb)));
            const double padlon = std::max(pad / cos(maxabs * RAD), pad * aspect);
            lspan = lon_span + 2.0 * padlon;
            l0 = lon0 - padlon;
            if (lspan >= 359.0) fl = true;
        }
        if (fl) {
            lspan = 360.0;
            l0 = -180.0;
            if (!north && !south) {
                if (latmin + latmax >= 0.0)
                    north = true;
                else
                    south = true;
            }
        }
        if (north) lb = 90.0;
        if (south) la = -90.0;
        la = std::max(la, -90.0);
        lb = std::min(lb, 90.0);
        full_lon = fl;
        G->lon0 = l0;
        G->lat0 = la;
        lon_span = fl ? 360.0 : lon_span;
        const double ncell = sqrt(lspan * (lb - la) / ((double)std::max(target, 1LL) * aspect));
        if (it < 2 && fabs(ncell - cell) > 1e-3 * cell) {
            cell = ncell;
            if (!fl) lon0 = lon0;  // unchanged: padding recomputed from the unpadded span
            continue;
        }
        long long W = std::max(1LL, (long long)ceil(lspan / (cell * aspect)));
        long long H = std::max(1LL, (long long)ceil((lb - la) / cell));
        W = std::min(W, 16384LL);
        H = std::min(H, 16384LL);
        if ((long long)W * H >= (long long)INDEX_MASK / 4) {
            set_error("exact index: top level too large");
            return GAHHG_ERR_CAPACITY;
        }
        G->W = (int)W;
        G->H = (int)H;
        G->dlon0 = lspan / (double)W;
        G->dlat0 = (lb - la) / (double)H;
        G->full_lon = full_lon;
        G->to_north = north;
        G->to_south = south;
        // cos(latitude) at the domain's equator-ward edge, rounded up
        const double la_eq = (la <= 0.0 && lb >= 0.0) ? 0.0 : std::min(fabs(la), fabs(lb));
        G->cap_cos = std::min(1.0, cos(la_eq * RAD) * (1.0 + 1e-9) + 1e-12);
        break;
    }
    return GAHHG_OK;
}

gahhg_status lattice_build(Grid* g)
{
    cudaStream_t s = g->stream;
    const Polygon* P = g->poly;
    const int n = P->pv_num;
    Lattice* L = new Lattice();
    g->lattice = L;
    // GAHHG_DEBUG: wall time of each phase (synchronising) on stderr
    const bool dbg = getenv("GAHHG_DEBUG") != nullptr;
    double tph = now_seconds();
    auto phase = [&](const char* name) {
        if (!dbg) return;
        cudaStreamSynchronize(s);
        const double t = now_seconds();
        fprintf(stderr, "lattice phase %-12s %9.3f ms\n", name, (t - tph) * 1e3);
        tph = t;
    };

    long long target = g->opts.lattice_top > 0 ? (long long)g->opts.lattice_top
                                                : std::min<long long>(std::max<long long>(8LL * n, 1024), 8LL << 20);
    GAHHG_TRY(compute_domain(P, target, &L->geo, s, g->device));
    phase("domain");
    const int W = L->geo.W, H = L->geo.H;
    L->K = g->opts.lattice_leaf > 0 ? g->opts.lattice_leaf : 8;
    L->maxlev = 9;
    static_assert(9 <= MAX_DESCENT, "the query's binary-fraction descent covers MAX_DESCENT levels");
    BuildView bv{L->geo, P->d_pv, P->d_pe, n};

    // exact label of the first level-0 center: from a point just left of an
    // outer edge, through the hubs whenever an arc would exceed ~84 degrees
    GAHHG_TRY(reference_point(g, L->x_in));
    int label = CELL_IN;
    {
        const NodeCap c00 = node_cap(L->geo, 0, 0, 0);
        std::vector<const double*> path;
        path.push_back(L->x_in);
        auto unit_dot = [](const double* a, const double* b) {
            return (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]) /
                   sqrt((a[0] * a[0] + a[1] * a[1] + a[2] * a[2]) * (b[0] * b[0] + b[1] * b[1] + b[2] * b[2]));
        };
        if (unit_dot(L->x_in, c00.R) < 0.1) {
            const int ha = nearest_hub(L->x_in), hb = nearest_hub(c00.R);
            path.push_back(HUBS[ha]);
            if ((ha ^ 1) == hb) path.push_back(HUBS[(ha + 2) % 6]);  // opposite hubs: go round
            if (hb != ha) path.push_back(HUBS[hb]);
        }
        path.push_back(c00.R);
        for (size_t k = 0; k + 1 < path.size(); k++) {
            int par;
            GAHHG_TRY(arc_parity_all(g, path[k], path[k + 1], &par, nullptr, nullptr));
            if (par < 0) {
                set_error("exact index: a hub or the origin center coincides with a polygon vertex");
                return GAHHG_ERR_STATE;
            }
            if (par) label = 3 - label;
        }
    }
    L->origin_label = label;

    phase("origin");
    std::vector<LevelBuf> lv(1);
    // ---------------- level 0 ----------------
    LevelBuf& l0 = lv[0];
    l0.nn = W * H;
    l0.gstart = 0;
    GAHHG_TRY(l0.cnt.reserve(l0.nn, s, false));
    GAHHG_TRY(l0.off.reserve(l0.nn, s, false));
    GAHHG_TRY(l0.cursor.reserve(l0.nn, s, false));
    GAHHG_CUDA_TRY(cudaMemsetAsync(l0.cnt.ptr, 0, sizeof(int) * l0.nn, s));
    GAHHG_CUDA_TRY(cudaMemsetAsync(l0.cursor.ptr, 0, sizeof(int) * l0.nn, s));
    // candidate boxes split into work items of bounded size, then the pair
    // tests over the items (count pass, scan, fill pass)
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
    DevArray<EdgeBox> boxes;
    DevArray<int> items, item_off;
    GAHHG_TRY(boxes.reserve(std::max(n, 1), s, false));
    GAHHG_TRY(items.reserve(std::max(n, 1), s, false));
    GAHHG_TRY(item_off.reserve(std::max(n, 1), s, false));
    unsigned long long* d_items64 = reinterpret_cast<unsigned long long*>(g->d_counts + 16);
    int* d_items = g->d_counts + 18;
    GAHHG_CUDA_TRY(cudaMemsetAsync(d_items64, 0, sizeof(unsigned long long), s));
    k_l0_box<<<blocks_for(n), TPB, 0, s>>>(bv, boxes.ptr, items.ptr, d_items64);
    GAHHG_TRY(scan_state_reserve(&g->scan_state, std::max(n, l0.nn)));
    GAHHG_TRY(scan_exclusive(items.ptr, item_off.ptr, n, d_items, g->scan_state, g->d_err, s));
    unsigned long long items64 = 0;
    GAHHG_CUDA_TRY(cudaMemcpyAsync(&items64, d_items64, sizeof(items64), cudaMemcpyDeviceToHost, s));
    GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
    if (items64 > (unsigned long long)INT_MAX) {
        set_error("exact index: %llu level-0 candidate work items exceed 2^31 (fewer top cells are needed)",
                  items64);
        return GAHHG_ERR_CAPACITY;
    }
    // the count pass's hits per item, so the fill pass does not test again
    DevArray<unsigned long long> hits;
    if (items64 <= L0_MASK_ITEMS) GAHHG_TRY(hits.reserve(std::max<unsigned long long>(items64, 1), s, false));
    const OneGeo one{L->geo};
    k_l0_expand<0><<<sms * 8, TPB, 0, s>>>(bv.pv, bv.pe, (long long)n, one, boxes.ptr, item_off.ptr, d_items,
                                            d_items64, l0.cnt.ptr, nullptr, nullptr, nullptr, hits.ptr);
    GAHHG_TRY(scan_exclusive(l0.cnt.ptr, l0.off.ptr, l0.nn, g->d_counts + 8, g->scan_state, g->d_err, s));
    int total = 0;
    GAHHG_CUDA_TRY(cudaMemcpyAsync(&total, g->d_counts + 8, sizeof(int), cudaMemcpyDeviceToHost, s));
    GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
    phase("l0 count");
    l0.npairs = total;
    GAHHG_TRY(l0.list.reserve(std::max(total, 1), s, false));
    k_l0_expand<1><<<sms * 8, TPB, 0, s>>>(bv.pv, bv.pe, (long long)n, one, boxes.ptr, item_off.ptr, d_items,
                                            d_items64, l0.cnt.ptr, l0.off.ptr, l0.cursor.ptr, l0.list.ptr, hits.ptr);
    hits.release();
    boxes.release();
    items.release();
    item_off.release();
    GAHHG_TRY(sort_lists(g, l0.cnt.ptr, l0.off.ptr, l0.nn, l0.list.ptr, sms, s));
    phase("l0 fill");
    GAHHG_TRY(l0.ix.reserve(l0.nn, s, false));
    GAHHG_TRY(l0.iy.reserve(l0.nn, s, false));
    k_l0_coords<<<blocks_for(l0.nn), TPB, 0, s>>>(W, l0.nn, l0.ix.ptr, l0.iy.ptr);

    // level-0 labels
    bool has_outside_label = false;
    uint8_t* d_outside = nullptr;
    int* d_bad = g->d_counts + 48;  // [0] coincidences, [1] nesting, [2] long lists
    GAHHG_CUDA_TRY(cudaMemsetAsync(d_bad, 0, 4 * sizeof(int), s));
    {
        DevArray<uint8_t> vpar, hpar;
        GAHHG_TRY(vpar.reserve((size_t)W * (H > 1 ? H - 1 : 1) + 1, s, false));
        GAHHG_TRY(hpar.reserve(W, s, false));
        GAHHG_TRY(l0.label.reserve(l0.nn, s, false));
        const long long nthreads = (long long)W * (H - 1) + W - 1;
        k_l0_neighbour_parity<<<blocks_for(nthreads), TPB, 0, s>>>(bv, l0.cnt.ptr, l0.off.ptr, l0.list.ptr, vpar.ptr,
                                                                   hpar.ptr, d_bad);
        int* d_origin = g->d_counts + 12;
        GAHHG_CUDA_TRY(cudaMemcpyAsync(d_origin, &L->origin_label, sizeof(int), cudaMemcpyHostToDevice, s));
        k_l0_labels<<<blocks_for(W), TPB, 0, s>>>(W, H, vpar.ptr, hpar.ptr, d_origin, l0.label.ptr);
        // label of the region outside the domain, from the nearest border cell
        const Geo& G0 = L->geo;
        int ix = 0, iy = 0, ox = 0, oy = 0;
        bool has_outside = true;
        if (!G0.full_lon) {
            ox = -1;
        } else if (!G0.to_south) {
            oy = -1;
        } else if (!G0.to_north) {
            iy = H - 1;
            oy = H;
        } else {
            has_outside = false;
        }
        uint8_t* d_out = reinterpret_cast<uint8_t*>(g->d_counts + 13);
        // read back with the build's last round trip
        has_outside_label = has_outside;
        d_outside = d_out;
        if (has_outside)
            k_outside_label<<<1, 1, 0, s>>>(bv, ix, iy, ox, oy, l0.cnt.ptr, l0.off.ptr, l0.list.ptr, l0.label.ptr,
                                            d_out, d_bad);
        else
            L->outside_label = CELL_UNDEFINED;
        vpar.release();
        hpar.release();
    }

    phase("l0 labels");
    // ---------------- refinement ----------------
    int gnext = l0.nn;
    for (int lvl = 0; lvl < L->maxlev; lvl++) {
        LevelBuf& pl = lv[lvl];
        GAHHG_TRY(pl.flag.reserve(pl.nn, s, false));
        GAHHG_TRY(pl.foff.reserve(pl.nn, s, false));
        k_refine_flags<<<blocks_for(pl.nn), TPB, 0, s>>>(pl.cnt.ptr, pl.nn, L->K, pl.flag.ptr);
        GAHHG_TRY(scan_state_reserve(&g->scan_state, pl.nn));
        GAHHG_TRY(scan_exclusive(pl.flag.ptr, pl.foff.ptr, pl.nn, g->d_counts + 9, g->scan_state, g->d_err, s));
        int nref = 0;
        GAHHG_CUDA_TRY(cudaMemcpyAsync(&nref, g->d_counts + 9, sizeof(int), cudaMemcpyDeviceToHost, s));
        GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
        if (getenv("GAHHG_DEBUG"))
            fprintf(stderr, "lattice level %d: %d cells, %d edge entries, %d split (W=%d H=%d K=%d)\n", lvl, pl.nn,
                    pl.npairs, nref, L->geo.W, L->geo.H, L->K);
        if (nref == 0) break;
        // Bounded refinement: a polygon whose edges fill an area densely (not
        // a curve) would need cells below the edge spacing everywhere.  Past
        // the budget the remaining cells stay leaves with more edges: the
        // labels are the same, the crossing loops longer.
        if ((long long)gnext + (long long)nref * FAN * FAN > NODE_BUDGET || 4LL * pl.npairs > PAIR_BUDGET) {
            if (getenv("GAHHG_DEBUG"))
                fprintf(stderr, "lattice level %d: refinement stopped at the node/entry budget\n", lvl);
            break;
        }
        lv.emplace_back();
        LevelBuf& cl = lv.back();
        LevelBuf& pp = lv[lvl];  // re-fetch after emplace_back
        cl.nn = nref * FAN * FAN;
        cl.gstart = gnext;
        GAHHG_TRY(pp.child_base.reserve(pp.nn, s, false));
        GAHHG_TRY(cl.ix.reserve(cl.nn, s, false));
        GAHHG_TRY(cl.iy.reserve(cl.nn, s, false));
        k_make_children<<<blocks_for(pp.nn), TPB, 0, s>>>(pp.flag.ptr, pp.foff.ptr, pp.nn, cl.gstart, pp.ix.ptr,
                                                          pp.iy.ptr, W, pp.child_base.ptr, cl.ix.ptr, cl.iy.ptr);
        GAHHG_TRY(pp.pair_node.reserve(std::max(pp.npairs, 1), s, false));
        k_fill_pair_node<<<blocks_for(pp.nn), TPB, 0, s>>>(pp.cnt.ptr, pp.off.ptr, pp.nn, pp.pair_node.ptr);
        GAHHG_TRY(cl.cnt.reserve(cl.nn, s, false));
        GAHHG_TRY(cl.off.reserve(cl.nn, s, false));
        GAHHG_TRY(cl.cursor.reserve(cl.nn, s, false));
        GAHHG_CUDA_TRY(cudaMemsetAsync(cl.cnt.ptr, 0, sizeof(int) * cl.nn, s));
        GAHHG_CUDA_TRY(cudaMemsetAsync(cl.cursor.ptr, 0, sizeof(int) * cl.nn, s));
        DevArray<double4> caps;
        DevArray<double2> capsb;
        DevArray<uint16_t> hit;
        GAHHG_TRY(caps.reserve(cl.nn, s, false));
        GAHHG_TRY(capsb.reserve(cl.nn, s, false));
        GAHHG_TRY(hit.reserve(std::max(pp.npairs, 1), s, false));
        k_child_caps<<<blocks_for(cl.nn), TPB, 0, s>>>(L->geo, lvl + 1, cl.nn, cl.ix.ptr, cl.iy.ptr, caps.ptr,
                                                       capsb.ptr);
        k_child_pairs_count<<<blocks_for(pp.npairs), TPB, 0, s>>>(
            bv, pp.npairs, pp.pair_node.ptr, pp.list.ptr, pp.child_base.ptr, caps.ptr, capsb.ptr, cl.gstart,
            cl.cnt.ptr, hit.ptr);
        GAHHG_TRY(scan_state_reserve(&g->scan_state, cl.nn));
        GAHHG_TRY(scan_exclusive(cl.cnt.ptr, cl.off.ptr, cl.nn, g->d_counts + 10, g->scan_state, g->d_err, s));
        int ctotal = 0;
        GAHHG_CUDA_TRY(cudaMemcpyAsync(&ctotal, g->d_counts + 10, sizeof(int), cudaMemcpyDeviceToHost, s));
        GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
        cl.npairs = ctotal;
        GAHHG_TRY(cl.list.reserve(std::max(ctotal, 1), s, false));
        k_child_pairs_fill<<<blocks_for(pp.npairs), TPB, 0, s>>>(pp.npairs, pp.pair_node.ptr, pp.list.ptr,
                                                                 pp.child_base.ptr, cl.gstart, hit.ptr, cl.off.ptr,
                                                                 cl.cursor.ptr, cl.list.ptr);
        hit.release();
        GAHHG_TRY(sort_lists(g, cl.cnt.ptr, cl.off.ptr, cl.nn, cl.list.ptr, sms, s));
        // child labels
        DevArray<int> child_parent;
        GAHHG_TRY(child_parent.reserve(cl.nn, s, false));
        k_child_parent<<<blocks_for(pp.nn), TPB, 0, s>>>(pp.child_base.ptr, pp.nn, cl.gstart, child_parent.ptr);
        GAHHG_TRY(cl.label.reserve(cl.nn, s, false));
        k_child_labels<<<blocks_for(cl.nn), TPB, 0, s>>>(bv, OneGeo{L->geo}, lvl, cl.nn, child_parent.ptr, cl.ix.ptr, cl.iy.ptr,
                                                         cl.cnt.ptr, cl.off.ptr, cl.list.ptr, caps.ptr, capsb.ptr,
                                                         pp.ix.ptr, pp.iy.ptr, pp.cnt.ptr, pp.off.ptr, pp.list.ptr,
                                                         pp.label.ptr, cl.label.ptr, d_bad);
        caps.release();
        capsb.release();
        child_parent.release();
        gnext += cl.nn;
    }
    L->nlev = (int)lv.size();
    L->nnodes = gnext;

    phase("refine");
    // ---------------- encode ----------------
    GAHHG_TRY(L->nodes.reserve(L->nnodes, s, false));
    std::vector<int> leaf_base(L->nlev), nleaf(L->nlev);
    std::vector<long long> rec_base(L->nlev);
    long long leaf_total = 0, rec_total = 0;
    std::vector<DevArray<int>> is_leaf(L->nlev), leaf_off(L->nlev), nrec(L->nlev), rec_off(L->nlev);
    // every level's leaf and record totals, read back together
    DevArray<int> d_tot;
    GAHHG_TRY(d_tot.reserve(2 * L->nlev, s, false));
    for (int lvl = 0; lvl < L->nlev; lvl++) {
        LevelBuf& b = lv[lvl];
        const int* cb = (lvl + 1 < L->nlev) ? b.child_base.ptr : nullptr;
        GAHHG_TRY(is_leaf[lvl].reserve(b.nn, s, false));
        GAHHG_TRY(leaf_off[lvl].reserve(b.nn, s, false));
        GAHHG_TRY(nrec[lvl].reserve(b.nn, s, false));
        GAHHG_TRY(rec_off[lvl].reserve(b.nn, s, false));
        k_leaf_flags<<<blocks_for(b.nn), TPB, 0, s>>>(b.nn, b.cnt.ptr, cb, is_leaf[lvl].ptr, nrec[lvl].ptr);
        GAHHG_TRY(scan_state_reserve(&g->scan_state, b.nn));
        GAHHG_TRY(scan_exclusive(is_leaf[lvl].ptr, leaf_off[lvl].ptr, b.nn, d_tot.ptr + 2 * lvl, g->scan_state,
                                 g->d_err, s));
        GAHHG_TRY(scan_exclusive(nrec[lvl].ptr, rec_off[lvl].ptr, b.nn, d_tot.ptr + 2 * lvl + 1, g->scan_state,
                                 g->d_err, s));
        // leaf indices are per level here: shifted by the level's leaf base below
        k_encode<<<blocks_for(b.nn), TPB, 0, s>>>(OneGeo{L->geo}, b.nn, b.gstart, b.cnt.ptr, cb, b.label.ptr, leaf_off[lvl].ptr,
                                                  L->nodes.ptr);
    }
    {
        std::vector<int> tot(2 * L->nlev);
        GAHHG_CUDA_TRY(cudaMemcpyAsync(tot.data(), d_tot.ptr, sizeof(int) * tot.size(), cudaMemcpyDeviceToHost, s));
        GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
        for (int lvl = 0; lvl < L->nlev; lvl++) {
            leaf_base[lvl] = (int)leaf_total;
            nleaf[lvl] = tot[2 * lvl];
            rec_base[lvl] = rec_total;
            leaf_total += tot[2 * lvl];
            rec_total += tot[2 * lvl + 1];
        }
    }
    d_tot.release();
    if (rec_total >= 0xFFFFFFFFll) {
        set_error("exact index: too many edge records");
        return GAHHG_ERR_CAPACITY;
    }
    // one spare leaf: the grouped pass 2 copies leaf records in 16-byte units
    GAHHG_TRY(L->leaves.reserve(leaf_total + 1, s, false));
    GAHHG_TRY(L->recs.reserve(std::max(rec_total, 1LL), s, false));
    GAHHG_TRY(L->eids.reserve(std::max(rec_total, 1LL), s, false));
    GAHHG_TRY(L->leafR.reserve(3 * (size_t)std::max(leaf_total, 1LL), s, false));
    GAHHG_TRY(L->ends.reserve(3 * (size_t)std::max(n, 1), s, false));
    L->nleaves = leaf_total;
    L->nrecs = rec_total;
    L->nedges = n;
    k_edge_ends<<<blocks_for(n), TPB, 0, s>>>(bv.pv, bv.pe, n, L->ends.ptr);
    for (int lvl = 0; lvl < L->nlev; lvl++) {
        LevelBuf& b = lv[lvl];
        k_leaf_records<<<blocks_for(b.nn), TPB, 0, s>>>(bv, OneGeo{L->geo}, lvl, b.nn, is_leaf[lvl].ptr, leaf_off[lvl].ptr,
                                                        rec_off[lvl].ptr, leaf_base[lvl], rec_base[lvl], b.ix.ptr,
                                                        b.iy.ptr, b.cnt.ptr, b.off.ptr, b.list.ptr, b.label.ptr,
                                                        L->leaves.ptr, L->recs.ptr, L->eids.ptr, L->leafR.ptr,
                                                        d_bad);
    }
    GAHHG_CUDA_TRY(cudaGetLastError());
    // leaf words were encoded with per-level leaf offsets; make them global
    for (int lvl = 1; lvl < L->nlev; lvl++) {
        if (leaf_base[lvl] == 0) continue;
        k_shift_leaf_words<<<blocks_for(lv[lvl].nn), TPB, 0, s>>>(L->nodes.ptr, lv[lvl].gstart, lv[lvl].nn, leaf_base[lvl]);
    }
    {
        // coarse summary: at most 65,536 cells (16 KB), staged in shared memory by the query
        int cs = 0;
        auto blocks = [&](int c) { return (long long)((W + (1 << c) - 1) >> c) * ((H + (1 << c) - 1) >> c); };
        while (blocks(cs) > 65536) cs++;
        const int CW = (W + (1 << cs) - 1) >> cs, CH = (H + (1 << cs) - 1) >> cs;
        L->cshift = cs;
        L->swords = (CW * CH + 15) / 16;
        GAHHG_TRY(L->summary.reserve(L->swords, s, false));
        GAHHG_CUDA_TRY(cudaMemsetAsync(L->summary.ptr, 0, sizeof(uint32_t) * L->swords, s));
        k_summary<<<blocks_for(CW * CH), TPB, 0, s>>>(L->nodes.ptr, W, H, cs, L->summary.ptr, CW * CH);
    }
    int bad[4];
    uint8_t ol = 0;
    GAHHG_CUDA_TRY(cudaMemcpyAsync(bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost, s));
    if (has_outside_label) GAHHG_CUDA_TRY(cudaMemcpyAsync(&ol, d_outside, 1, cudaMemcpyDeviceToHost, s));
    GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
    if (has_outside_label) L->outside_label = ol;
    phase("encode");
    for (auto& b : lv) b.release();
    for (int lvl = 0; lvl < L->nlev; lvl++) {
        is_leaf[lvl].release();
        leaf_off[lvl].release();
        nrec[lvl].release();
        rec_off[lvl].release();
    }
    if (bad[0] || bad[1] || bad[2]) {
        set_error("exact index: %d center/vertex coincidences, %d cap nesting violations, %d oversize leaves",
                  bad[0], bad[1], bad[2]);
        return GAHHG_ERR_DEVICE;
    }
    GAHHG_TRY(check_device_errors(g, "exact index build"));
    return GAHHG_OK;
}

gahhg_status lattice_query_with(const QueryView& Q, const double* d_lonlat, long long n, uint8_t* d_labels,
                                int precision, cudaStream_t s, uint64_t* d_counters, uint32_t* queue,
                                unsigned int* qcount, long long chunk, int device, const Tiers* tiers,
                                const PartScratch* part = nullptr, const LeafSortScratch* lsort = nullptr);

// The locate arithmetic of a view from its level-0 grid.
static void set_view_geo(QueryView& Q, const Geo& g)
{
    Q.W = g.W;
    Q.H = g.H;
    Q.Wd = (double)g.W;
    Q.Hd = (double)g.H;
    Q.su_lon = 1.0 / g.dlon0;
    Q.su_lat = 1.0 / g.dlat0;
    Q.u0 = -g.lon0 * Q.su_lon;
    Q.v0 = -(g.lat0 + 90.0) * Q.su_lat;
    Q.U360 = 360.0 * Q.su_lon;
    Q.full_lon = g.full_lon;
    Q.to_north = g.to_north;
    Q.to_south = g.to_south;
}

// Coarse summary shape of a level-0 grid: cells of 2^cshift x 2^cshift top
// cells, at most 65,536 of them (16 KB of 2-bit codes).
static void summary_shape(int W, int H, int* cshift, int* CW, int* CH)
{
    int cs = 0;
    auto blocks = [&](int c) { return (long long)((W + (1 << c) - 1) >> c) * ((H + (1 << c) - 1) >> c); };
    while (blocks(cs) > 65536) cs++;
    *cshift = cs;
    *CW = (W + (1 << cs) - 1) >> cs;
    *CH = (H + (1 << cs) - 1) >> cs;
}

QueryView make_view(const Grid* g)
{
    const Lattice* L = g->lattice;
    QueryView Q;
    set_view_geo(Q, L->geo);
    Q.outside = KIND_PURE | (uint32_t)L->outside_label;
    Q.nodes = L->nodes.ptr;
    Q.leaves = L->leaves.ptr;
    Q.recs = L->recs.ptr;
    Q.eids = L->eids.ptr;
    Q.ends = L->ends.ptr;
    Q.leafR = L->leafR.ptr;
    Q.pv = g->poly->d_pv;
    Q.pe = g->poly->d_pe;
    Q.cshift = L->cshift;
    Q.CW = (L->geo.W + (1 << L->cshift) - 1) >> L->cshift;
    Q.swords = L->swords;
    Q.summary = L->summary.ptr;
    // windows of about PART_BYTES of the records the tiers gather per leaf
    const long long tier_bytes = L->nrecs * (long long)(sizeof(float4) + sizeof(uint32_t)) +
                                 L->nleaves * (long long)(sizeof(LeafRec) + 3 * sizeof(double));
    Q.nparts = (int)std::min<long long>(PART_MAX, std::max<long long>(1, (tier_bytes + PART_BYTES - 1) / PART_BYTES));
    if (L->nleaves < 2 * PART_MAX) Q.nparts = 1;
    Q.part_scale = Q.nparts > 1 ? (float)((double)Q.nparts / (double)L->nleaves) : 0.0f;
    return Q;
}

// ------------------------------------------------------ group build host --

struct GroupIndex {
    int count = 0;
    DevArray<D3> pv;        // the group's vertices, polygon after polygon
    DevArray<int> pe;       // its edges (group vertex indices)
    DevArray<uint32_t> nodes;
    DevArray<LeafRec> leaves;
    DevArray<float4> recs;
    DevArray<uint32_t> eids;
    DevArray<double2> ends;
    DevArray<double> leafR;
    DevArray<uint32_t> summary;
    std::vector<QueryView> views;  // per polygon
    std::vector<int> swords;
    long long nnodes = 0, nleaves = 0, nrecs = 0, nedges = 0;
    void release()
    {
        pv.release();
        pe.release();
        nodes.release();
        leaves.release();
        recs.release();
        eids.release();
        ends.release();
        leafR.release();
        summary.release();
    }
};

void group_free(GroupIndex* G)
{
    if (!G) return;
    G->release();
    delete G;
}

void group_view_write(const GroupIndex* G, int i, void* dst) { memcpy(dst, &G->views[i], sizeof(QueryView)); }
long long group_summary_words(const GroupIndex* G, int i) { return G->swords[i]; }
long long group_bytes(const GroupIndex* G)
{
    return G->nnodes * (long long)sizeof(uint32_t) + G->nleaves * (long long)(sizeof(LeafRec) + 3 * sizeof(double)) +
           G->nrecs * (long long)(sizeof(float4) + sizeof(uint32_t)) + G->nedges * 3 * (long long)sizeof(double2);
}

namespace {

// host array -> device array on s (the device array is reserved here)
template <class T>
gahhg_status upload(DevArray<T>& d, const std::vector<T>& h, cudaStream_t s)
{
    GAHHG_TRY(d.reserve(std::max<size_t>(h.size(), 1), s, false));
    if (!h.empty()) GAHHG_CUDA_TRY(cudaMemcpyAsync(d.ptr, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, s));
    return GAHHG_OK;
}

}  // namespace

// Exact indexes of polys[0 .. count) built together on stream s (g carries
// the device, the scratch counts and error word and the scan state).  The
// steps and their order follow lattice_build; see the group kernels above.
gahhg_status lattice_build_group(Grid* g, Polygon* const* polys, int count, const int* top_cells,
                                 const int* leaf_edges, GroupIndex** out)
{
    cudaStream_t s = g->stream;
    const int np = count;
    // GAHHG_DEBUG: wall time of each phase (synchronising) on stderr
    const bool dbg = getenv("GAHHG_DEBUG") != nullptr;
    double tph = now_seconds();
    auto phase = [&](const char* name) {
        if (!dbg) return;
        cudaStreamSynchronize(s);
        const double t = now_seconds();
        fprintf(stderr, "group phase %-12s %9.3f ms (%d polygons)\n", name, (t - tph) * 1e3, np);
        tph = t;
    };
    GroupIndex* GI = new GroupIndex();
    *out = GI;
    GI->count = np;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);

    // ---- edges and vertices of the group
    std::vector<long long> ebase(np + 1, 0), vbase(np + 1, 0);
    std::vector<int> nouter(np);
    for (int p = 0; p < np; p++) {
        const Polygon* P = polys[p];
        ebase[p + 1] = ebase[p] + P->pv_num;
        vbase[p + 1] = vbase[p] + (long long)P->pv.size();
        nouter[p] = P->ring_start.size() > 1 ? P->ring_start[1] : P->pv_num;
    }
    const long long ne = ebase[np], nvx = vbase[np];
    if (ne >= INT_MAX / 2 || nvx >= INT_MAX) {
        set_error("exact index group: %lld edges exceed the group limit", ne);
        return GAHHG_ERR_CAPACITY;
    }
    GI->nedges = ne;
    GAHHG_TRY(GI->pv.reserve(std::max(nvx, 1LL), s, false));
    GAHHG_TRY(GI->pe.reserve(std::max(2 * ne, 1LL), s, false));
    for (int p = 0; p < np; p++) {
        const Polygon* P = polys[p];
        if (P->pv_num == 0) continue;
        GAHHG_CUDA_TRY(cudaMemcpyAsync(GI->pv.ptr + vbase[p], P->pv.data(), sizeof(D3) * P->pv.size(),
                                       cudaMemcpyHostToDevice, s));
        GAHHG_CUDA_TRY(cudaMemcpyAsync(GI->pe.ptr + 2 * ebase[p], P->pe.data(), sizeof(int) * 2 * P->pv_num,
                                       cudaMemcpyHostToDevice, s));
    }
    DevArray<long long> d_ebase, d_vbase;
    DevArray<int> epoly, d_nouter;
    GAHHG_TRY(upload(d_ebase, ebase, s));
    GAHHG_TRY(upload(d_vbase, vbase, s));
    GAHHG_TRY(upload(d_nouter, nouter, s));
    GAHHG_TRY(epoly.reserve(std::max(ne, 1LL), s, false));
    kb_edges<<<(int)((ne + TPB - 1) / TPB), TPB, 0, s>>>(d_ebase.ptr, d_vbase.ptr, np, ne, epoly.ptr, GI->pe.ptr);
    const D3* pv = GI->pv.ptr;
    const int* pe = GI->pe.ptr;
    BuildView bv{Geo{}, pv, pe, (int)ne};

    phase("upload");
    // ---- domains (one scan for every polygon, one round trip)
    std::vector<PolyGeo> pg(np);
    std::vector<long long> tops(np + 1, 0);
    {
        std::vector<DomainOut> h(np);
        for (auto& d : h) {
            memset(&d, 0, sizeof d);
            d.latmin = ~0ull;
        }
        DevArray<DomainOut> d;
        GAHHG_TRY(upload(d, h, s));
        const int grid = (int)std::max(1LL, std::min<long long>(sms * 8LL, (ne + TPB - 1) / TPB));
        kb_domain_scan<<<grid, TPB, 0, s>>>(pv, pe, ne, epoly.ptr, d.ptr);
        GAHHG_CUDA_TRY(cudaMemcpyAsync(h.data(), d.ptr, sizeof(DomainOut) * np, cudaMemcpyDeviceToHost, s));
        GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
        d.release();
        // the level-0 grids on host threads (a polygon's takes tens of microseconds)
        std::vector<gahhg_status> st(np, GAHHG_OK);
        std::vector<std::string> msg(np);
        auto geo_range = [&](int p0, int p1) {
            for (int p = p0; p < p1; p++) {
                const Polygon* P = polys[p];
                const long long n = P->pv_num;
                const long long target = top_cells && top_cells[p] > 0
                                             ? (long long)top_cells[p]
                                             : std::min<long long>(std::max<long long>(8LL * n, 1024), 8LL << 20);
                st[p] = geo_from_scan(h[p], P, target, &pg[p].g);
                if (st[p] != GAHHG_OK) msg[p] = last_error();
            }
        };
        const int nt = std::max(1, std::min({np / 16, 16, (int)std::max(1u, std::thread::hardware_concurrency())}));
        if (nt == 1) {
            geo_range(0, np);
        } else {
            std::vector<std::thread> th;
            for (int t = 0; t < nt; t++) th.emplace_back(geo_range, (int)((long long)np * t / nt), (int)((long long)np * (t + 1) / nt));
            for (auto& t : th) t.join();
        }
        for (int p = 0; p < np; p++) {
            if (st[p] != GAHHG_OK) {
                set_error("polygon %d: %s", p, msg[p].c_str());
                return st[p];
            }
            pg[p].K = leaf_edges && leaf_edges[p] > 0 ? leaf_edges[p] : 8;
            pg[p].e0 = (int)ebase[p];
            pg[p].top = tops[p];
            tops[p + 1] = tops[p] + (long long)pg[p].g.W * pg[p].g.H;
        }
    }
    const long long n0 = tops[np];
    if (n0 >= NODE_BUDGET) {
        set_error("exact index group: %lld level-0 cells exceed the node budget", n0);
        return GAHHG_ERR_CAPACITY;
    }
    DevArray<PolyGeo> d_pg;
    DevArray<long long> d_tops;
    GAHHG_TRY(upload(d_pg, pg, s));
    GAHHG_TRY(upload(d_tops, tops, s));

    phase("domain");
    // ---- exact label of every polygon's first level-0 center
    DevArray<int> origin;
    GAHHG_TRY(origin.reserve(np, s, false));
    kb_origin<<<np, ORIGIN_TPB, 0, s>>>(pv, pe, d_pg.ptr, d_ebase.ptr, d_nouter.ptr, origin.ptr);

    phase("origin");
    // ---- level 0: candidate boxes in work items, pair tests, lists
    std::vector<LevelBuf> lv(1);
    LevelBuf& l0 = lv[0];
    l0.nn = (int)n0;
    l0.gstart = 0;
    GAHHG_TRY(l0.cnt.reserve(l0.nn, s, false));
    GAHHG_TRY(l0.off.reserve(l0.nn, s, false));
    GAHHG_TRY(l0.cursor.reserve(l0.nn, s, false));
    GAHHG_CUDA_TRY(cudaMemsetAsync(l0.cnt.ptr, 0, sizeof(int) * l0.nn, s));
    GAHHG_CUDA_TRY(cudaMemsetAsync(l0.cursor.ptr, 0, sizeof(int) * l0.nn, s));
    {
        DevArray<EdgeBox> boxes;
        DevArray<int> items, item_off;
        GAHHG_TRY(boxes.reserve(std::max(ne, 1LL), s, false));
        GAHHG_TRY(items.reserve(std::max(ne, 1LL), s, false));
        GAHHG_TRY(item_off.reserve(std::max(ne, 1LL), s, false));
        unsigned long long* d_items64 = reinterpret_cast<unsigned long long*>(g->d_counts + 16);
        int* d_items = g->d_counts + 18;
        GAHHG_CUDA_TRY(cudaMemsetAsync(d_items64, 0, sizeof(unsigned long long), s));
        kb_l0_box<<<(int)((ne + TPB - 1) / TPB), TPB, 0, s>>>(pv, pe, ne, epoly.ptr, d_pg.ptr, boxes.ptr, items.ptr,
                                                              d_items64);
        GAHHG_TRY(scan_state_reserve(&g->scan_state, (int)std::max<long long>(ne, l0.nn)));
        GAHHG_TRY(scan_exclusive(items.ptr, item_off.ptr, (int)ne, d_items, g->scan_state, g->d_err, s));
        unsigned long long items64 = 0;
        GAHHG_CUDA_TRY(cudaMemcpyAsync(&items64, d_items64, sizeof(items64), cudaMemcpyDeviceToHost, s));
        GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
        if (items64 > (unsigned long long)INT_MAX) {
            set_error("exact index group: %llu level-0 candidate work items exceed 2^31", items64);
            return GAHHG_ERR_CAPACITY;
        }
        DevArray<unsigned long long> hits;
        if (items64 <= L0_MASK_ITEMS) GAHHG_TRY(hits.reserve(std::max<unsigned long long>(items64, 1), s, false));
        const EdgeGeoTable eg{d_pg.ptr, epoly.ptr};
        k_l0_expand<0><<<sms * 8, TPB, 0, s>>>(pv, pe, ne, eg, boxes.ptr, item_off.ptr, d_items, d_items64,
                                                l0.cnt.ptr, nullptr, nullptr, nullptr, hits.ptr);
        GAHHG_TRY(scan_exclusive(l0.cnt.ptr, l0.off.ptr, l0.nn, g->d_counts + 8, g->scan_state, g->d_err, s));
        int total = 0;
        GAHHG_CUDA_TRY(cudaMemcpyAsync(&total, g->d_counts + 8, sizeof(int), cudaMemcpyDeviceToHost, s));
        GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
        l0.npairs = total;
        GAHHG_TRY(l0.list.reserve(std::max(total, 1), s, false));
        k_l0_expand<1><<<sms * 8, TPB, 0, s>>>(pv, pe, ne, eg, boxes.ptr, item_off.ptr, d_items, d_items64,
                                                l0.cnt.ptr, l0.off.ptr, l0.cursor.ptr, l0.list.ptr, hits.ptr);
        hits.release();
    }
    phase("l0 pairs");
    GAHHG_TRY(sort_lists(g, l0.cnt.ptr, l0.off.ptr, l0.nn, l0.list.ptr, sms, s));
    GAHHG_TRY(l0.ix.reserve(l0.nn, s, false));
    GAHHG_TRY(l0.iy.reserve(l0.nn, s, false));
    GAHHG_TRY(l0.poly.reserve(l0.nn, s, false));
    kb_l0_coords<<<blocks_for(l0.nn), TPB, 0, s>>>(d_tops.ptr, np, d_pg.ptr, l0.nn, l0.ix.ptr, l0.iy.ptr,
                                                   l0.poly.ptr);

    phase("l0 sort");
    // ---- level-0 labels and each polygon's label outside its domain
    int* d_bad = g->d_counts + 48;  // [0] coincidences, [1] nesting, [2] long lists
    GAHHG_CUDA_TRY(cudaMemsetAsync(d_bad, 0, 4 * sizeof(int), s));
    DevArray<uint8_t> outl;
    GAHHG_TRY(outl.reserve(np, s, false));
    {
        std::vector<long long> pb(np + 1, 0), cb(np + 1, 0);
        std::vector<int4> oxy(np);
        for (int p = 0; p < np; p++) {
            const Geo& G0 = pg[p].g;
            const int W = G0.W, H = G0.H;
            pb[p + 1] = pb[p] + (long long)W * (H - 1) + (W - 1);
            cb[p + 1] = cb[p] + W;
            // the region outside the domain, from the nearest border cell
            int ix = 0, iy = 0, ox = 0, oy = 0;
            if (!G0.full_lon) {
                ox = -1;
            } else if (!G0.to_south) {
                oy = -1;
            } else if (!G0.to_north) {
                iy = H - 1;
                oy = H;
            } else {
                ox = INT_MIN;  // no outside region
            }
            oxy[p] = make_int4(ix, iy, ox, oy);
        }
        DevArray<long long> d_pb, d_cb;
        DevArray<int4> d_oxy;
        DevArray<uint8_t> par;
        GAHHG_TRY(upload(d_pb, pb, s));
        GAHHG_TRY(upload(d_cb, cb, s));
        GAHHG_TRY(upload(d_oxy, oxy, s));
        GAHHG_TRY(par.reserve(std::max(pb[np], 1LL), s, false));
        GAHHG_TRY(l0.label.reserve(l0.nn, s, false));
        if (pb[np] > 0)
            kb_l0_neighbour_parity<<<(int)((pb[np] + TPB - 1) / TPB), TPB, 0, s>>>(
                pv, pe, d_pg.ptr, d_pb.ptr, np, l0.cnt.ptr, l0.off.ptr, l0.list.ptr, par.ptr, d_bad);
        kb_l0_labels<<<(int)((cb[np] + TPB - 1) / TPB), TPB, 0, s>>>(d_pg.ptr, d_cb.ptr, d_pb.ptr, np, par.ptr,
                                                                      origin.ptr, l0.label.ptr);
        kb_outside_label<<<(np + TPB - 1) / TPB, TPB, 0, s>>>(pv, pe, d_pg.ptr, np, d_oxy.ptr, l0.cnt.ptr,
                                                               l0.off.ptr, l0.list.ptr, l0.label.ptr, outl.ptr, d_bad);
        par.release();
        d_pb.release();
        d_cb.release();
        d_oxy.release();
    }

    phase("l0 labels");
    // ---- refinement, every polygon's level at once
    const int maxlev = 9;
    long long gnext = l0.nn;
    for (int lvl = 0; lvl < maxlev; lvl++) {
        LevelBuf& pl = lv[lvl];
        GAHHG_TRY(pl.flag.reserve(pl.nn, s, false));
        GAHHG_TRY(pl.foff.reserve(pl.nn, s, false));
        kb_refine_flags<<<blocks_for(pl.nn), TPB, 0, s>>>(pl.cnt.ptr, pl.poly.ptr, d_pg.ptr, pl.nn, pl.flag.ptr);
        GAHHG_TRY(scan_state_reserve(&g->scan_state, pl.nn));
        GAHHG_TRY(scan_exclusive(pl.flag.ptr, pl.foff.ptr, pl.nn, g->d_counts + 9, g->scan_state, g->d_err, s));
        int nref = 0;
        GAHHG_CUDA_TRY(cudaMemcpyAsync(&nref, g->d_counts + 9, sizeof(int), cudaMemcpyDeviceToHost, s));
        GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
        if (nref == 0) break;
        // the budgets hold for the whole group (a polygon built alone keeps its
        // own); past them the remaining cells stay leaves with more edges
        if (gnext + (long long)nref * FAN * FAN > NODE_BUDGET || 4LL * pl.npairs > PAIR_BUDGET) break;
        lv.emplace_back();
        LevelBuf& cl = lv.back();
        LevelBuf& pp = lv[lvl];  // re-fetch after emplace_back
        cl.nn = nref * FAN * FAN;
        cl.gstart = (int)gnext;
        GAHHG_TRY(pp.child_base.reserve(pp.nn, s, false));
        GAHHG_TRY(cl.ix.reserve(cl.nn, s, false));
        GAHHG_TRY(cl.iy.reserve(cl.nn, s, false));
        GAHHG_TRY(cl.poly.reserve(cl.nn, s, false));
        kb_make_children<<<blocks_for(pp.nn), TPB, 0, s>>>(pp.flag.ptr, pp.foff.ptr, pp.nn, cl.gstart, pp.ix.ptr,
                                                           pp.iy.ptr, pp.poly.ptr, pp.child_base.ptr, cl.ix.ptr,
                                                           cl.iy.ptr, cl.poly.ptr);
        GAHHG_TRY(pp.pair_node.reserve(std::max(pp.npairs, 1), s, false));
        k_fill_pair_node<<<blocks_for(pp.nn), TPB, 0, s>>>(pp.cnt.ptr, pp.off.ptr, pp.nn, pp.pair_node.ptr);
        GAHHG_TRY(cl.cnt.reserve(cl.nn, s, false));
        GAHHG_TRY(cl.off.reserve(cl.nn, s, false));
        GAHHG_TRY(cl.cursor.reserve(cl.nn, s, false));
        GAHHG_CUDA_TRY(cudaMemsetAsync(cl.cnt.ptr, 0, sizeof(int) * cl.nn, s));
        GAHHG_CUDA_TRY(cudaMemsetAsync(cl.cursor.ptr, 0, sizeof(int) * cl.nn, s));
        DevArray<double4> caps;
        DevArray<double2> capsb;
        DevArray<uint16_t> hit;
        GAHHG_TRY(caps.reserve(cl.nn, s, false));
        GAHHG_TRY(capsb.reserve(cl.nn, s, false));
        GAHHG_TRY(hit.reserve(std::max(pp.npairs, 1), s, false));
        kb_child_caps<<<blocks_for(cl.nn), TPB, 0, s>>>(d_pg.ptr, lvl + 1, cl.nn, cl.ix.ptr, cl.iy.ptr, cl.poly.ptr,
                                                        caps.ptr, capsb.ptr);
        k_child_pairs_count<<<blocks_for(pp.npairs), TPB, 0, s>>>(bv, pp.npairs, pp.pair_node.ptr, pp.list.ptr,
                                                                  pp.child_base.ptr, caps.ptr, capsb.ptr, cl.gstart,
                                                                  cl.cnt.ptr, hit.ptr);
        GAHHG_TRY(scan_state_reserve(&g->scan_state, cl.nn));
        GAHHG_TRY(scan_exclusive(cl.cnt.ptr, cl.off.ptr, cl.nn, g->d_counts + 10, g->scan_state, g->d_err, s));
        int ctotal = 0;
        GAHHG_CUDA_TRY(cudaMemcpyAsync(&ctotal, g->d_counts + 10, sizeof(int), cudaMemcpyDeviceToHost, s));
        GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
        cl.npairs = ctotal;
        GAHHG_TRY(cl.list.reserve(std::max(ctotal, 1), s, false));
        k_child_pairs_fill<<<blocks_for(pp.npairs), TPB, 0, s>>>(pp.npairs, pp.pair_node.ptr, pp.list.ptr,
                                                                 pp.child_base.ptr, cl.gstart, hit.ptr, cl.off.ptr,
                                                                 cl.cursor.ptr, cl.list.ptr);
        hit.release();
        GAHHG_TRY(sort_lists(g, cl.cnt.ptr, cl.off.ptr, cl.nn, cl.list.ptr, sms, s));
        DevArray<int> child_parent;
        GAHHG_TRY(child_parent.reserve(cl.nn, s, false));
        k_child_parent<<<blocks_for(pp.nn), TPB, 0, s>>>(pp.child_base.ptr, pp.nn, cl.gstart, child_parent.ptr);
        GAHHG_TRY(cl.label.reserve(cl.nn, s, false));
        k_child_labels<<<blocks_for(cl.nn), TPB, 0, s>>>(bv, TableGeo{d_pg.ptr, pp.poly.ptr}, lvl, cl.nn,
                                                         child_parent.ptr, cl.ix.ptr, cl.iy.ptr, cl.cnt.ptr,
                                                         cl.off.ptr, cl.list.ptr, caps.ptr, capsb.ptr, pp.ix.ptr,
                                                         pp.iy.ptr, pp.cnt.ptr, pp.off.ptr, pp.list.ptr,
                                                         pp.label.ptr, cl.label.ptr, d_bad);
        caps.release();
        capsb.release();
        child_parent.release();
        gnext += cl.nn;
    }
    const int nlev = (int)lv.size();
    GI->nnodes = gnext;

    phase("refine");
    // ---- encode: node words, leaf records, summaries
    GAHHG_TRY(GI->nodes.reserve(std::max(GI->nnodes, 1LL), s, false));
    std::vector<int> leaf_base(nlev);
    std::vector<long long> rec_base(nlev);
    long long leaf_total = 0, rec_total = 0;
    std::vector<DevArray<int>> is_leaf(nlev), leaf_off(nlev), nrec(nlev), rec_off(nlev);
    DevArray<int> d_tot;
    GAHHG_TRY(d_tot.reserve(2 * nlev, s, false));
    for (int lvl = 0; lvl < nlev; lvl++) {
        LevelBuf& b = lv[lvl];
        const int* cbase = (lvl + 1 < nlev) ? b.child_base.ptr : nullptr;
        GAHHG_TRY(is_leaf[lvl].reserve(b.nn, s, false));
        GAHHG_TRY(leaf_off[lvl].reserve(b.nn, s, false));
        GAHHG_TRY(nrec[lvl].reserve(b.nn, s, false));
        GAHHG_TRY(rec_off[lvl].reserve(b.nn, s, false));
        k_leaf_flags<<<blocks_for(b.nn), TPB, 0, s>>>(b.nn, b.cnt.ptr, cbase, is_leaf[lvl].ptr, nrec[lvl].ptr);
        GAHHG_TRY(scan_state_reserve(&g->scan_state, b.nn));
        GAHHG_TRY(scan_exclusive(is_leaf[lvl].ptr, leaf_off[lvl].ptr, b.nn, d_tot.ptr + 2 * lvl, g->scan_state,
                                 g->d_err, s));
        GAHHG_TRY(scan_exclusive(nrec[lvl].ptr, rec_off[lvl].ptr, b.nn, d_tot.ptr + 2 * lvl + 1, g->scan_state,
                                 g->d_err, s));
        k_encode<<<blocks_for(b.nn), TPB, 0, s>>>(TableGeo{d_pg.ptr, b.poly.ptr}, b.nn, b.gstart, b.cnt.ptr, cbase,
                                                  b.label.ptr, leaf_off[lvl].ptr, GI->nodes.ptr);
    }
    {
        std::vector<int> tot(2 * nlev);
        GAHHG_CUDA_TRY(cudaMemcpyAsync(tot.data(), d_tot.ptr, sizeof(int) * tot.size(), cudaMemcpyDeviceToHost, s));
        GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
        for (int lvl = 0; lvl < nlev; lvl++) {
            leaf_base[lvl] = (int)leaf_total;
            rec_base[lvl] = rec_total;
            leaf_total += tot[2 * lvl];
            rec_total += tot[2 * lvl + 1];
        }
    }
    d_tot.release();
    if (rec_total >= 0xFFFFFFFFll || leaf_total >= (long long)INDEX_MASK) {
        set_error("exact index group: too many leaves or edge records");
        return GAHHG_ERR_CAPACITY;
    }
    GAHHG_TRY(GI->leaves.reserve(leaf_total + 1, s, false));
    GAHHG_TRY(GI->recs.reserve(std::max(rec_total, 1LL), s, false));
    GAHHG_TRY(GI->eids.reserve(std::max(rec_total, 1LL), s, false));
    GAHHG_TRY(GI->leafR.reserve(3 * (size_t)std::max(leaf_total, 1LL), s, false));
    GAHHG_TRY(GI->ends.reserve(3 * (size_t)std::max(ne, 1LL), s, false));
    GI->nleaves = leaf_total;
    GI->nrecs = rec_total;
    k_edge_ends<<<(int)((ne + TPB - 1) / TPB), TPB, 0, s>>>(pv, pe, (int)ne, GI->ends.ptr);
    for (int lvl = 0; lvl < nlev; lvl++) {
        LevelBuf& b = lv[lvl];
        k_leaf_records<<<blocks_for(b.nn), TPB, 0, s>>>(bv, TableGeo{d_pg.ptr, b.poly.ptr}, lvl, b.nn,
                                                        is_leaf[lvl].ptr, leaf_off[lvl].ptr, rec_off[lvl].ptr,
                                                        leaf_base[lvl], rec_base[lvl], b.ix.ptr, b.iy.ptr, b.cnt.ptr,
                                                        b.off.ptr, b.list.ptr, b.label.ptr, GI->leaves.ptr,
                                                        GI->recs.ptr, GI->eids.ptr, GI->leafR.ptr, d_bad);
    }
    GAHHG_CUDA_TRY(cudaGetLastError());
    for (int lvl = 1; lvl < nlev; lvl++) {
        if (leaf_base[lvl] == 0) continue;
        k_shift_leaf_words<<<blocks_for(lv[lvl].nn), TPB, 0, s>>>(GI->nodes.ptr, lv[lvl].gstart, lv[lvl].nn,
                                                                  leaf_base[lvl]);
    }
    // coarse summaries, each polygon's from a 16-byte aligned word
    std::vector<long long> sc(np + 1, 0), soff(np + 1, 0);
    std::vector<int> cshift(np);
    GI->swords.resize(np);
    for (int p = 0; p < np; p++) {
        int cs, CW, CH;
        summary_shape(pg[p].g.W, pg[p].g.H, &cs, &CW, &CH);
        cshift[p] = cs;
        GI->swords[p] = (CW * CH + 15) / 16;
        sc[p + 1] = sc[p] + (long long)CW * CH;
        soff[p + 1] = soff[p] + ((GI->swords[p] + 3) & ~3);
    }
    {
        DevArray<long long> d_sc, d_soff;
        DevArray<int> d_cshift;
        GAHHG_TRY(upload(d_sc, sc, s));
        GAHHG_TRY(upload(d_soff, soff, s));
        GAHHG_TRY(upload(d_cshift, cshift, s));
        // 1,024 spare words: a bulk copy of a summary reads up to its 16-byte multiple
        GAHHG_TRY(GI->summary.reserve(soff[np] + 1024, s, false));
        GAHHG_CUDA_TRY(cudaMemsetAsync(GI->summary.ptr, 0, sizeof(uint32_t) * (soff[np] + 1024), s));
        kb_summary<<<(int)((sc[np] + TPB - 1) / TPB), TPB, 0, s>>>(GI->nodes.ptr, d_pg.ptr, d_sc.ptr, d_cshift.ptr,
                                                                   d_soff.ptr, np, GI->summary.ptr);
        d_sc.release();
        d_soff.release();
        d_cshift.release();
    }
    phase("encode");
    // ---- the build's last round trip: failures, origins, outside labels
    int bad[4];
    std::vector<int> h_origin(np);
    std::vector<uint8_t> h_out(np);
    GAHHG_CUDA_TRY(cudaMemcpyAsync(bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost, s));
    GAHHG_CUDA_TRY(cudaMemcpyAsync(h_origin.data(), origin.ptr, sizeof(int) * np, cudaMemcpyDeviceToHost, s));
    GAHHG_CUDA_TRY(cudaMemcpyAsync(h_out.data(), outl.ptr, np, cudaMemcpyDeviceToHost, s));
    GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
    for (auto& b : lv) b.release();
    for (int lvl = 0; lvl < nlev; lvl++) {
        is_leaf[lvl].release();
        leaf_off[lvl].release();
        nrec[lvl].release();
        rec_off[lvl].release();
    }
    for (int p = 0; p < np; p++) {
        if (h_origin[p] == 0) {
            set_error("exact index: polygon %d: no outer-ring edge gives a reference point", p);
            return GAHHG_ERR_STATE;
        }
        if (h_origin[p] < 0) {
            set_error("exact index: polygon %d: a hub or the origin center coincides with a polygon vertex", p);
            return GAHHG_ERR_STATE;
        }
    }
    if (bad[0] || bad[1] || bad[2]) {
        set_error("exact index group: %d center/vertex coincidences, %d cap nesting violations, %d oversize leaves",
                  bad[0], bad[1], bad[2]);
        return GAHHG_ERR_DEVICE;
    }
    GAHHG_TRY(check_device_errors(g, "exact index group build"));
    // ---- every polygon's query view into the group's arrays
    GI->views.resize(np);
    for (int p = 0; p < np; p++) {
        QueryView& Q = GI->views[p];
        memset(&Q, 0, sizeof Q);
        set_view_geo(Q, pg[p].g);
        Q.outside = KIND_PURE | (uint32_t)h_out[p];
        Q.nodes = GI->nodes.ptr + pg[p].top;
        Q.leaves = GI->leaves.ptr;
        Q.recs = GI->recs.ptr;
        Q.eids = GI->eids.ptr;
        Q.ends = GI->ends.ptr;
        Q.leafR = GI->leafR.ptr;
        Q.pv = pv;
        Q.pe = pe;
        Q.cshift = cshift[p];
        Q.CW = (pg[p].g.W + (1 << cshift[p]) - 1) >> cshift[p];
        Q.swords = GI->swords[p];
        Q.summary = GI->summary.ptr + soff[p];
        Q.nparts = 1;  // the leaf-window order of single-polygon queries is not used by batches
        Q.part_scale = 0.0f;
    }
    return GAHHG_OK;
}

// Points per pass; the pass-2 queue holds one 4-byte index per point.
constexpr long long QUERY_CHUNK = 1LL << 27;

gahhg_status lattice_query(Grid* g, const double* d_lonlat, size_t n, uint8_t* d_labels, int precision,
                           cudaStream_t s, uint64_t* d_counters)
{
    if (n == 0) return GAHHG_OK;
    const QueryView Q = make_view(g);
    const long long chunk = std::min<long long>((long long)n, QUERY_CHUNK);
    // Words: [pass-2 queue: chunk][control: 192 (queue fill at +32, tier
    // counters at +33..35, window-order flag at +36, entries per window at
    // +64, windows' cursors at +128)][pass-2 leaf words: chunk][tier-2 queue]
    // [its leaf words][tier-3 queue][its leaf words][tier-2 masks][queue in
    // window order: points, leaf words (chunk each)].
    // One memset per pass clears the control words from the queue fill on.
    // [leaf order only: entries per leaf: nb][leaf starts: nb + 1][tile
    // sums][ranks: chunk].
    unsigned int cap2 = 0, cap3 = 0;
    tier_caps(chunk, &cap2, &cap3);
    const long long order = knob(GAHHG_KNOB_GROUPED_PASS2);
    const bool windows = order == 1 && Q.nparts > 1 && chunk >= PART_MIN_QUEUE;
    const bool leaves = (order == 2 || order == 3) && chunk >= PART_MIN_QUEUE && g->lattice->nleaves > 0 &&
                        g->lattice->nleaves < (1LL << 30);
    const int nb = leaves ? (int)g->lattice->nleaves + 1 : 0;
    const int tiles = (nb + LS_TILE - 1) / LS_TILE;
    const size_t l1_at = (size_t)chunk + 192;
    // even, so that the leaf order's (point, leaf word) pairs are 8-byte aligned
    const size_t sorted_at = (l1_at + (size_t)chunk + 3 * (size_t)cap2 + 2 * (size_t)cap3 + 1) & ~(size_t)1;
    const size_t ls_at = sorted_at + 2 * (size_t)chunk;
    const size_t words = windows ? ls_at : leaves ? ls_at + 2 * (size_t)nb + 1 + tiles + (size_t)chunk : sorted_at;
    uint32_t* queue = nullptr;
    GAHHG_TRY(pool_alloc((void**)&queue, sizeof(uint32_t) * words, g->device, s));
    unsigned int* qcount = (unsigned int*)(queue + chunk + 32);
    Tiers T;
    T.cnt = qcount + 1;
    T.l1 = queue + l1_at;
    T.q2 = T.l1 + chunk;
    T.l2 = T.q2 + cap2;
    T.q3 = T.l2 + cap2;
    T.l3 = T.q3 + cap3;
    T.m2 = T.l3 + cap3;
    T.cap2 = cap2;
    T.cap3 = cap3;
    PartScratch W;
    W.done = qcount + 4;
    W.total = queue + chunk + 64;
    W.cursor = queue + chunk + 128;
    W.spts = queue + sorted_at;
    W.sleaf = queue + sorted_at + chunk;
    W.np = Q.nparts;
    W.scale = Q.part_scale;
    LeafSortScratch LS;
    LS.done = qcount + 4;
    LS.sent = (uint2*)(queue + sorted_at);
    LS.cnt = queue + ls_at;
    LS.start = LS.cnt + nb;
    LS.tsum = LS.start + nb + 1;
    LS.rank = LS.tsum + tiles;
    LS.nb = nb;
    LS.tiles = tiles;
    LS.stage = order == 3;
    const gahhg_status st = lattice_query_with(Q, d_lonlat, (long long)n, d_labels, precision, s, d_counters,
                                               queue, qcount, chunk, g->device, &T, windows ? &W : nullptr,
                                               leaves ? &LS : nullptr);
    cudaFreeAsync(queue, s);
    return st;
}

// tiers == nullptr: one pass-2 launch with escalations inline (no queues
// beyond the pass-2 queue); else qcount[1..3] are the tier counters.
gahhg_status lattice_query_with(const QueryView& Q, const double* d_lonlat, long long n, uint8_t* d_labels,
                                int precision, cudaStream_t s, uint64_t* d_counters, uint32_t* queue,
                                unsigned int* qcount, long long chunk, int device, const Tiers* tiers,
                                const PartScratch* part, const LeafSortScratch* lsort)
{
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    unsigned long long* ctr = (unsigned long long*)d_counters;
    for (long long off = 0; off < n; off += chunk) {
        const int m = (int)std::min<long long>(chunk, n - off);
        const double2* ll = (const double2*)d_lonlat + off;
        // the queue fill, the tier counters and, when ordering by window, the
        // flag, the counts and the cursors (the control words run up to them)
        const size_t zero_words = part ? (size_t)(part->cursor + PART_MAX - qcount) : lsort ? 5 : (tiers ? 4 : 1);
        GAHHG_CUDA_TRY(cudaMemsetAsync(qcount, 0, sizeof(unsigned int) * zero_words, s));
        if (lsort) GAHHG_CUDA_TRY(cudaMemsetAsync(lsort->cnt, 0, sizeof(unsigned int) * lsort->nb, s));
        const long long tiles = ((long long)m + TPB * LOC_UNROLL - 1) / (TPB * LOC_UNROLL);
        const int grid = (int)std::min<long long>(tiles, (long long)sms * 8);
        uint32_t* leafq = tiers ? tiers->l1 : nullptr;
        const int polls = (int)knob(GAHHG_KNOB_STAGING_POLL_LIMIT);
        auto kl = ctr ? k_locate<true> : k_locate<false>;
        kl<<<grid, TPB, summary_bytes(Q.swords), s>>>(ll, m, d_labels + off, Q, queue, leafq, qcount, ctr, polls);
        if (tiers && part) {
            // the pass-1 queue in window order, then the tiers over it
            launch_dependent_tpb(k_part_count, sms * 4, P_TPB, s, (const uint32_t*)tiers->l1,
                                 (const unsigned int*)qcount, *part);
            launch_dependent_tpb(k_part_scatter, sms * 4, P_TPB, s, (const uint32_t*)queue,
                                 (const uint32_t*)tiers->l1, (const unsigned int*)qcount, *part);
            Tiers T = *tiers;
            T.spts = part->spts;
            T.sleaf = part->sleaf;
            T.sorted = part->done;
            leaf_tiers_launch(OneView{Q}, ll, d_labels + off, queue, qcount, T, precision, ctr, sms, s);
        } else if (tiers && lsort) {
            // the pass-1 queue in leaf order, then the tiers over it
            const uint32_t* l1 = tiers->l1;
            const unsigned int* qc = qcount;
            launch_dependent_tpb(k_ls_count, sms * 8, LS_TPB, s, l1, qc, *lsort);
            launch_dependent_tpb(k_ls_tile_sums, std::min(lsort->tiles, sms * 8), LS_TPB, s, qc, *lsort);
            launch_dependent_tpb(k_ls_scan, std::min(lsort->tiles, sms * 8), LS_TPB, s, qc, *lsort);
            launch_dependent_tpb(k_ls_scatter, sms * 8, LS_TPB, s, (const uint32_t*)queue, l1, qc, *lsort);
            Tiers T = *tiers;
            T.spts = (const uint32_t*)lsort->sent;
            T.sleaf = T.spts + 1;
            T.sstride = 2;
            T.sorted = lsort->done;
            leaf_tiers_launch(OneView{Q}, ll, d_labels + off, queue, qcount, T, precision, ctr, sms, s,
                              lsort->stage);
        } else if (tiers) {
            leaf_tiers_launch(OneView{Q}, ll, d_labels + off, queue, qcount, *tiers, precision, ctr, sms, s);
        }
        else if (precision == GAHHG_QUERY_FP64_FILTER)
            k_leaf<false><<<sms * 4, TPB, 0, s>>>(ll, d_labels + off, Q, queue, qcount, ctr);
        else
            k_leaf<true><<<sms * 4, TPB, 0, s>>>(ll, d_labels + off, Q, queue, qcount, ctr);
        GAHHG_CUDA_TRY(cudaGetLastError());
    }
    return GAHHG_OK;
}

// ------------------------------------------------- allocation-free query --
//
// The same two passes as lattice_query, with the pass-2 queue in a fixed
// array in device memory instead of memory taken from the pool, for callers
// that must not allocate (see gahhg_query_device_noalloc in include/gahhg.h).
// Every device that loads this library reserves the array until the process
// exits.  All calls share it: calls that overlap on the GPU race.

constexpr long long NOALLOC_MAX_POINTS = 1LL << 21;  // 2,097,152 points per call
static __device__ __align__(256) uint32_t g_noalloc_queue[NOALLOC_MAX_POINTS + 64];

long long lattice_noalloc_max_points() { return NOALLOC_MAX_POINTS; }

// Device address of the array on the current device (the caller has made
// g->device current).  In host code `g_noalloc_queue` names a host-side
// stand-in, never the device array, so the address is asked of the runtime.
// It is looked up on every call rather than cached: after cudaDeviceReset
// (or any other teardown of the primary context) the module is loaded again
// and the array may sit at another address.  The lookup allocates nothing;
// the first one on a device loads the module there, which is why the first
// call on a device should come before any stream capture.
static gahhg_status noalloc_queue_address(int device, uint32_t** out)
{
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_queue);
    if (e != cudaSuccess || !p) {
        set_error("cudaGetSymbolAddress(g_noalloc_queue) on device %d: %s", device, cudaGetErrorString(e));
        return GAHHG_ERR_CUDA;
    }
    *out = (uint32_t*)p;
    return GAHHG_OK;
}

gahhg_status lattice_query_noalloc(Grid* g, const double* d_lonlat, size_t n, uint8_t* d_labels, int precision,
                                   cudaStream_t s)
{
    if ((long long)n > NOALLOC_MAX_POINTS) {
        set_error("gahhg_query_device_noalloc: %zu points exceed the fixed maximum of %lld per call", n,
                  NOALLOC_MAX_POINTS);
        return GAHHG_ERR_CAPACITY;
    }
    if ((uintptr_t)d_lonlat & 15u) {
        set_error("exact queries read lon/lat in 16-byte units: the device buffer must be 16-byte aligned");
        return GAHHG_ERR_ARG;
    }
    uint32_t* queue = nullptr;
    GAHHG_TRY(noalloc_queue_address(g->device, &queue));
    if (n == 0) return GAHHG_OK;
    const QueryView Q = make_view(g);
    // the queue count lives after the queue; lattice_query_with zeroes it before each pass
    unsigned int* qcount = (unsigned int*)(queue + NOALLOC_MAX_POINTS + 32);
    return lattice_query_with(Q, d_lonlat, (long long)n, d_labels, precision, s, nullptr, queue, qcount,
                              NOALLOC_MAX_POINTS, g->device, nullptr);
}

// ------------------------------------------------------- batch launcher --

size_t lattice_view_bytes() { return sizeof(QueryView); }
size_t batch_chunk_bytes() { return sizeof(BatchChunk); }

void lattice_view_write(const Grid* g, void* dst)
{
    const QueryView q = make_view(g);
    memcpy(dst, &q, sizeof(q));
}

long long lattice_summary_words(const Grid* g) { return g->lattice ? g->lattice->swords : 0; }

gahhg_status lattice_staging_fallbacks(int device, unsigned long long* out)
{
    GAHHG_CUDA_TRY(cudaSetDevice(device));
    unsigned int v = 0;
    GAHHG_CUDA_TRY(cudaMemcpyFromSymbol(&v, g_tma_timeouts, sizeof(v)));
    *out = v;
    return GAHHG_OK;
}

// Chunks of at most `chunk_points` points, segment after segment.
// A segment's chunks hold at least 16 points per word of its summary, so
// staging the summary costs at most a quarter byte per point.
void batch_write_chunks(const long long* offsets, int nseg, int chunk_points, const int* swords, const int* seg_view,
                        void* out, int* nchunks)
{
    BatchChunk* v = (BatchChunk*)out;
    int n = 0;
    for (int p = 0; p < nseg; p++) {
        const long long step = std::max<long long>(chunk_points, 16LL * (swords ? swords[p] : 0));
        for (long long a = offsets[p]; a < offsets[p + 1]; a += step) {
            BatchChunk c;
            c.view = seg_view ? seg_view[p] : p;
            c.start = a;
            c.count = (int)std::min<long long>(step, offsets[p + 1] - a);
            if (v) v[n] = c;
            n++;
        }
    }
    *nchunks = n;
}

size_t batch_chunk_count_bound(long long points, int nseg, int chunk_points)
{
    return (size_t)(points / std::max(chunk_points, 1)) + (size_t)nseg + 1;
}

void batch_make_chunks(const long long* offsets, int nseg, int chunk_points, const int* swords, const int* seg_view,
                       std::vector<uint8_t>& out, int* nchunks)
{
    int n = 0;
    batch_write_chunks(offsets, nseg, chunk_points, swords, seg_view, nullptr, &n);
    out.resize((size_t)n * sizeof(BatchChunk));
    batch_write_chunks(offsets, nseg, chunk_points, swords, seg_view, out.data(), nchunks);
}

// Launches the batch locate instance of shape `shape` (statistics on when
// `ctr` is set).
template <int I>
static void batch_locate_launch(int shape, int grid, cudaStream_t s, const QueryView* views, const BatchChunk* chunks,
                                int nchunks, unsigned int* next_chunk, const double2* ll, uint8_t* out,
                                uint32_t* queue, uint32_t* leafq, unsigned int* qcount, unsigned long long* ctr,
                                int polls)
{
    if constexpr (I < BATCH_NSHAPES) {
        if (shape != I) {
            batch_locate_launch<I + 1>(shape, grid, s, views, chunks, nchunks, next_chunk, ll, out, queue, leafq,
                                       qcount, ctr, polls);
            return;
        }
        constexpr int U = BATCH_SHAPES[I].unroll, B = BATCH_SHAPES[I].blocks;
        if (ctr)
            k_batch_locate<true, U, B><<<grid, TPB, 0, s>>>(views, chunks, nchunks, next_chunk, ll, out, queue, leafq,
                                                            qcount, ctr, polls);
        else
            k_batch_locate<false, U, B><<<grid, TPB, 0, s>>>(views, chunks, nchunks, next_chunk, ll, out, queue,
                                                             leafq, qcount, ctr, polls);
    }
}

int batch_shape_count() { return BATCH_NSHAPES; }

bool batch_shape_info(int shape, int* points_per_thread, int* blocks_per_sm)
{
    if (shape < 0 || shape >= BATCH_NSHAPES) return false;
    if (points_per_thread) *points_per_thread = BATCH_SHAPES[shape].unroll;
    if (blocks_per_sm) *blocks_per_sm = BATCH_SHAPES[shape].blocks;
    return true;
}

size_t batch_queue_words(long long queue_cap)
{
    unsigned int cap2 = 0, cap3 = 0;
    tier_caps(queue_cap, &cap2, &cap3);
    return 2 * ((size_t)queue_cap + cap2 + cap3) + cap2;
}

// counters: [0] queue count, [1] next chunk, [2..4] tier counters.  The
// queue holds batch_queue_words(queue_cap) words: the pass-2 queue and its
// leaf words, then the escalation queues, each followed by its leaf words.  Everything is enqueued on `s` (no allocation, no host
// synchronisation), so it can be captured in a graph.
gahhg_status batch_query_launch(const void* d_views, const void* d_chunks, int nchunks, const double* d_lonlat,
                                uint8_t* d_labels, int precision, uint32_t* queue, long long queue_cap,
                                unsigned int* counters, uint64_t* d_stats, cudaStream_t s, int device,
                                bool zero_counters, int shape)
{
    if (nchunks == 0) return GAHHG_OK;
    static std::atomic<int> sms_cache[64];
    int sms = (device >= 0 && device < 64) ? sms_cache[device].load(std::memory_order_relaxed) : 0;
    if (!sms) {
        sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        if (device >= 0 && device < 64) sms_cache[device].store(sms, std::memory_order_relaxed);
    }
    const QueryView* views = (const QueryView*)d_views;
    const BatchChunk* chunks = (const BatchChunk*)d_chunks;
    unsigned long long* ctr = (unsigned long long*)d_stats;
    if (zero_counters) GAHHG_CUDA_TRY(cudaMemsetAsync(counters, 0, 5 * sizeof(unsigned int), s));
    Tiers T;
    tier_caps(queue_cap, &T.cap2, &T.cap3);
    T.l1 = queue + queue_cap;
    T.q2 = T.l1 + queue_cap;
    T.l2 = T.q2 + T.cap2;
    T.q3 = T.l2 + T.cap2;
    T.l3 = T.q3 + T.cap3;
    T.m2 = T.l3 + T.cap3;
    T.cnt = counters + 2;
    const int polls = (int)knob(GAHHG_KNOB_STAGING_POLL_LIMIT);
    if (shape < 0 || shape >= BATCH_NSHAPES) shape = 0;
    const int grid = std::min(nchunks, sms * BATCH_SHAPES[shape].blocks);  // persistent: every block resident
    batch_locate_launch<0>(shape, grid, s, views, chunks, nchunks, counters + 1, (const double2*)d_lonlat, d_labels,
                           queue, T.l1, counters, ctr, polls);
    leaf_tiers_launch(ChunkViews{views, chunks, nchunks}, (const double2*)d_lonlat, d_labels, queue, counters, T,
                      precision, ctr, sms, s);
    GAHHG_CUDA_TRY(cudaGetLastError());
    return GAHHG_OK;
}

}  // namespace gahhg
