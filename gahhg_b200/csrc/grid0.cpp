// grid0.cpp - the 42-cell level-0 grid of the hexagon hierarchy.
//
// The reference obtains this grid from initgrid0 (declared at
// source/common.h:201, consumed at source/GPISPAHHG.cu:1962-1973) whose only
// implementation is a closed library, so the construction here is this
// project's own, built to the contract its consumers impose:
//   - 42 cells (the loops `i < 42` at source/GPISPAHHG.cu:1177,1439);
//   - 80 vertices, 240 borders (the initial capacities at :1958-1960), i.e.
//     the dual of the frequency-2 geodesic icosahedron: 12 pentagons and
//     30 hexagons;
//   - each border runs counter-clockwise around its cell seen from outside,
//     with inward normal normalize(v0 x (v1 - v0)) (inside <=> n.p >= -eps,
//     :208-224), partner = twin half-edge, subcell/upcell = -1, type = 0.
//
// Construction: icosahedron with vertices at both poles and rings at
// latitude +-atan(1/2) (upper ring at lon 0,72,..; lower ring at 36,108,..),
// written with algebraic sines and cosines of multiples of 36 degrees so that
// only IEEE-exact sqrt is involved; one midpoint subdivision; the dual grid
// (one vertex per triangle = normalised vertex sum, one cell per point, ring
// ordered counter-clockwise starting at the lowest triangle index).
#include "gahhg_internal.h"

#include <algorithm>
#include <cstring>

namespace gahhg {

void build_grid0(std::vector<D3>& V, std::vector<Border>& B, std::vector<Cell>& C)
{
    const double r5 = sqrt(5.0);
    const double h = 1.0 / r5, rr = 2.0 / r5;
    const double c36 = (1.0 + r5) / 4.0, s36 = sqrt(10.0 - 2.0 * r5) / 4.0;
    const double c72 = (r5 - 1.0) / 4.0, s72 = sqrt(10.0 + 2.0 * r5) / 4.0;
    // sin/cos of lon 0,72,144,216,288 (upper ring) and 36,108,180,252,324 (lower)
    const double us[5] = {0.0, s72, s36, -s36, -s72}, uc[5] = {1.0, c72, -c36, -c36, c72};
    const double ls[5] = {s36, s72, 0.0, -s72, -s36}, lc[5] = {c36, -c72, -1.0, -c72, c36};

    std::vector<D3> pts;
    pts.reserve(42);
    pts.push_back(normalize(d3(0.0, 1.0, 0.0)));
    for (int i = 0; i < 5; i++) pts.push_back(normalize(d3(rr * us[i], h, rr * uc[i])));
    for (int i = 0; i < 5; i++) pts.push_back(normalize(d3(rr * ls[i], -h, rr * lc[i])));
    pts.push_back(normalize(d3(0.0, -1.0, 0.0)));

    int face[20][3];
    for (int i = 0; i < 5; i++) {
        const int j = (i + 1) % 5;
        const int f[4][3] = {{0, 1 + i, 1 + j}, {1 + i, 6 + i, 1 + j}, {1 + j, 6 + i, 6 + j}, {11, 6 + j, 6 + i}};
        for (int q = 0; q < 4; q++) std::memcpy(face[5 * q + i], f[q], sizeof(f[q]));
    }

    std::vector<int> mid_lo, mid_hi;
    auto mid = [&](int a, int b) -> int {
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        for (size_t k = 0; k < mid_lo.size(); k++)
            if (mid_lo[k] == lo && mid_hi[k] == hi) return 12 + (int)k;
        mid_lo.push_back(lo);
        mid_hi.push_back(hi);
        pts.push_back(normalize(pts[a] + pts[b]));
        return (int)pts.size() - 1;
    };

    int tri[80][3];
    for (int f = 0; f < 20; f++) {
        const int a = face[f][0], b = face[f][1], c = face[f][2];
        const int ab = mid(a, b), bc = mid(b, c), ca = mid(c, a);
        const int t[4][3] = {{a, ab, ca}, {ab, b, bc}, {ca, bc, c}, {ab, bc, ca}};
        std::memcpy(tri[4 * f], t, sizeof(t));
    }

    V.resize(80);
    for (int t = 0; t < 80; t++) V[t] = normalize((pts[tri[t][0]] + pts[tri[t][1]]) + pts[tri[t][2]]);

    B.clear();
    C.clear();
    for (int k = 0; k < 42; k++) {
        std::vector<int> around;
        for (int t = 0; t < 80; t++)
            if (tri[t][0] == k || tri[t][1] == k || tri[t][2] == k) around.push_back(t);
        // order by angle about pts[k], first triangle at angle 0
        const D3 c = pts[k];
        const D3 d0 = V[around[0]];
        const D3 e1 = normalize(d0 - c * dot(c, d0));
        const D3 e2 = cross(c, e1);
        std::vector<std::pair<double, int>> by_angle;
        for (int t : around) {
            double a = (t == around[0]) ? 0.0 : atan2(dot(e2, V[t]), dot(e1, V[t]));
            if (a < 0) a += 2.0 * M_PI;
            by_angle.push_back({a, t});
        }
        std::sort(by_angle.begin(), by_angle.end());
        const int n = (int)by_angle.size();
        Cell cell;
        cell.bstart = (int)B.size();
        cell.bnum = n;
        cell.rstart = -1;
        cell.rnum = 0;
        cell.upcell = -1;
        cell.subcell = -1;
        cell.type = CELL_UNDEFINED;
        for (int i = 0; i < n; i++) {
            Border b;
            b.parent = k;
            b.partner = -1;
            b.v[0] = by_angle[i].second;
            b.v[1] = by_angle[(i + 1) % n].second;
            b.subcell = -1;
            b.id = i;
            const D3 nn = edge_normal(V[b.v[0]], V[b.v[1]]);
            b.n[0] = nn.x;
            b.n[1] = nn.y;
            b.n[2] = nn.z;
            B.push_back(b);
        }
        C.push_back(cell);
    }
    for (size_t i = 0; i < B.size(); i++)
        for (size_t j = 0; j < B.size(); j++)
            if (B[j].v[0] == B[i].v[1] && B[j].v[1] == B[i].v[0]) {
                B[i].partner = (int)j;
                break;
            }
}

}  // namespace gahhg
