// ref_grid0.cpp - initgrid0() for the CPU build of the reference.
//
// TEST INFRASTRUCTURE.  The reference declares initgrid0 in source/common.h:201
// and ships it only inside a closed static library, so its exact vertices are
// unknown.  This file builds the level-0 grid the way this project defines it
// (the product builds the same grid in gahhg_b200/csrc/grid0.cpp; a test
// compares the two bit for bit):
//
//   1. icosahedron with vertices at both poles, upper ring at lon 0,72,..,288
//      and lower ring at lon 36,108,..,324 (latitudes +-atan(1/2)), written
//      with algebraic sines/cosines of multiples of 36 degrees;
//   2. one frequency-2 subdivision (edge midpoints, normalised) -> 42 points,
//      80 triangles;
//   3. the dual: one grid vertex per triangle (normalised vertex sum), one
//      cell per point, 12 pentagons and 30 hexagons, 240 half-edge borders.
//
// It satisfies the contract the reference's consumers impose
// (source/GPISPAHHG.cu:1949-1973, 1177, 1439, 208-224): 42 cells; 80
// vertices / 240 borders / 42 cells fit the initial capacities; each border's
// v[0]->v[1] runs counter-clockwise around its cell seen from outside, its
// normal is normalize(v0 x (v1 - v0)) and points into the cell; partner is the
// twin half-edge; subcell = upcell = -1; type = 0.
#include "refshim.h"
#include "common.h"

#include <algorithm>
#include <vector>

namespace {

struct V3 {
    double x, y, z;
};

V3 add(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
double dotp(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 crossp(V3 a, V3 b)
{
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
V3 unit(V3 a)
{
    double t = 1.0 / sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
    return V3{a.x * t, a.y * t, a.z * t};
}

}  // namespace

void initgrid0(myArray<mydouble3>* vout, myArray<AHHGBorder>* bout, myArray<AHHGCell>* cout_)
{
    const double r5 = sqrt(5.0);
    const double h = 1.0 / r5, rr = 2.0 / r5;
    const double c36 = (1.0 + r5) / 4.0, s36 = sqrt(10.0 - 2.0 * r5) / 4.0;
    const double c72 = (r5 - 1.0) / 4.0, s72 = sqrt(10.0 + 2.0 * r5) / 4.0;
    // (sin, cos) of 0,72,144,216,288 and of 36,108,180,252,324 degrees
    const double up_s[5] = {0.0, s72, s36, -s36, -s72};
    const double up_c[5] = {1.0, c72, -c36, -c36, c72};
    const double lo_s[5] = {s36, s72, 0.0, -s72, -s36};
    const double lo_c[5] = {c36, -c72, -1.0, -c72, c36};

    std::vector<V3> P;
    P.push_back(unit(V3{0.0, 1.0, 0.0}));
    for (int i = 0; i < 5; i++) P.push_back(unit(V3{rr * up_s[i], h, rr * up_c[i]}));
    for (int i = 0; i < 5; i++) P.push_back(unit(V3{rr * lo_s[i], -h, rr * lo_c[i]}));
    P.push_back(unit(V3{0.0, -1.0, 0.0}));

    int F[20][3];
    for (int i = 0; i < 5; i++) {
        int j = (i + 1) % 5;
        F[i][0] = 0;           F[i][1] = 1 + i;      F[i][2] = 1 + j;
        F[5 + i][0] = 1 + i;   F[5 + i][1] = 6 + i;  F[5 + i][2] = 1 + j;
        F[10 + i][0] = 1 + j;  F[10 + i][1] = 6 + i; F[10 + i][2] = 6 + j;
        F[15 + i][0] = 11;     F[15 + i][1] = 6 + j; F[15 + i][2] = 6 + i;
    }

    // midpoints, numbered in first-seen order over faces and their edges
    std::vector<std::pair<int, int>> mid_key;
    auto midpoint = [&](int a, int b) {
        int lo = std::min(a, b), hi = std::max(a, b);
        for (size_t k = 0; k < mid_key.size(); k++)
            if (mid_key[k].first == lo && mid_key[k].second == hi) return 12 + (int)k;
        mid_key.push_back({lo, hi});
        P.push_back(unit(add(P[a], P[b])));
        return 12 + (int)mid_key.size() - 1;
    };
    int T[80][3];
    for (int f = 0; f < 20; f++) {
        int a = F[f][0], b = F[f][1], c = F[f][2];
        int mab = midpoint(a, b), mbc = midpoint(b, c), mca = midpoint(c, a);
        int t[4][3] = {{a, mab, mca}, {mab, b, mbc}, {mca, mbc, c}, {mab, mbc, mca}};
        for (int q = 0; q < 4; q++)
            for (int e = 0; e < 3; e++) T[4 * f + q][e] = t[q][e];
    }

    std::vector<V3> D(80);
    for (int t = 0; t < 80; t++) D[t] = unit(add(add(P[T[t][0]], P[T[t][1]]), P[T[t][2]]));

    // rings: triangles around each point, counter-clockwise seen from outside,
    // starting with the lowest triangle index
    std::vector<std::vector<int>> ring(42);
    for (int k = 0; k < 42; k++) {
        std::vector<int> adj;
        for (int t = 0; t < 80; t++)
            if (T[t][0] == k || T[t][1] == k || T[t][2] == k) adj.push_back(t);
        V3 c = P[k];
        V3 d0 = D[adj[0]];
        V3 e1 = unit(sub(d0, V3{c.x * dotp(c, d0), c.y * dotp(c, d0), c.z * dotp(c, d0)}));
        V3 e2 = crossp(c, e1);
        std::vector<std::pair<double, int>> ang;
        for (int t : adj) {
            double a = atan2(dotp(e2, D[t]), dotp(e1, D[t]));
            if (t == adj[0]) a = 0.0;
            if (a < 0) a += 2.0 * M_PI;
            ang.push_back({a, t});
        }
        std::sort(ang.begin(), ang.end());
        for (auto& pr : ang) ring[k].push_back(pr.second);
    }

    for (int t = 0; t < 80; t++) vout->addElem(mydouble3(D[t].x, D[t].y, D[t].z));

    int bstart = 0;
    for (int k = 0; k < 42; k++) {
        int n = (int)ring[k].size();
        for (int i = 0; i < n; i++) {
            AHHGBorder b;
            b.parent = k;
            b.partner = -1;
            b.v[0] = ring[k][i];
            b.v[1] = ring[k][(i + 1) % n];
            b.subcell = -1;
            b.id = i;
            // device_getENormal (source/GPISPAHHG.cu:18-25)
            V3 e0 = D[b.v[0]];
            V3 e1 = sub(D[b.v[1]], D[b.v[0]]);
            V3 nn = unit(crossp(e0, e1));
            b.n[0] = nn.x;
            b.n[1] = nn.y;
            b.n[2] = nn.z;
            bout->addElem(b);
        }
        AHHGCell c;
        c.bstart = bstart;
        c.bnum = n;
        c.rstart = -1;
        c.rnum = 0;
        c.upcell = -1;
        c.subcell = -1;
        c.type = 0;
        cout_->addElem(c);
        bstart += n;
    }
    for (int i = 0; i < bout->curNum; i++) {
        for (int j = 0; j < bout->curNum; j++) {
            if (bout->elem[j].v[0] == bout->elem[i].v[1] && bout->elem[j].v[1] == bout->elem[i].v[0]) {
                bout->elem[i].partner = j;
                break;
            }
        }
    }
}
