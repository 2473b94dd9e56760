// walk.cuh - FP64 predicates of the hexagon hierarchy and the edge walk.
//
// Reference semantics, operation for operation (all epsilons included):
//   device_isPointInsideCell   source/GPISPAHHG.cu:208-224
//   device_isEdgeBorderInter   source/GPISPAHHG.cu:226-284
//   device_getSegExitBorder    source/GPISPAHHG.cu:286-348
//   the walk loop              source/GPISPAHHG.cu:1208-1287 (mark),
//                              :734-816 (count), :870-953 (write)
// Differences, all in cases where the reference would read outside its
// arrays or never finish: a missing partner (-1), a cell index outside the
// grid, a walk that returns to a state it was in before (the next step
// depends only on the current cell and the border it entered by, so such a
// walk would repeat forever; Brent's cycle test finds it within a few times
// the cycle's length) or a walk longer than the step limit (GridView::
// walk_limit, default WALK_STEP_LIMIT, gahhg_set_knob) ends the walk and
// is counted in DeviceErrors instead of reading garbage or spinning.  A walk
// that ends in the reference never repeats a state, so none of these changes
// a walk the reference completes.
#pragma once

#include "gahhg_internal.h"

namespace gahhg {

constexpr int WALK_STEP_LIMIT = 1 << 16;

struct GridView {
    const D3* V;
    Border* B;
    Cell* C;
    int nb;  // borders in use (valid indices [0, nb))
    int nc;  // cells in use
    int walk_limit = WALK_STEP_LIMIT;  // steps before a walk gives up
};

__device__ __forceinline__ int inside_cell(D3 p, int cid, const GridView& g)
{
    if (cid < 0 || cid >= g.nc) return -1;
    const int bs = g.C[cid].bstart, bn = g.C[cid].bnum;
    for (int i = 0; i < bn; i++) {
        const double* n = g.B[bs + i].n;
        double ret = n[0] * p.x + n[1] * p.y + n[2] * p.z;
        if (ret < -POSITION_EPSILON) return -1;
    }
    return cid;
}

__device__ __forceinline__ int edge_border_inter(D3 p0, D3 p1, D3 v0, D3 v1, int& reserved)
{
    D3 n0 = normalize(cross(v0, v1 - v0));
    double r0 = dot(n0, p0), r1 = dot(n0, p1);
    D3 n1 = normalize(cross(p0, p1 - p0));
    double r2 = dot(n1, v0), r3 = dot(n1, v1);

    if (equ_zero(r0) && equ_zero(r1)) return INTER_OVERLAP;
    const bool sep23 = (less_zero(r2) && less_zero(r3)) || (gre_zero(r2) && gre_zero(r3));
    const bool sep01 = (less_zero(r0) && less_zero(r1)) || (gre_zero(r0) && gre_zero(r1));
    if (!sep23 && equ_zero(r0)) {
        reserved = 0;
        return INTER_T1;
    }
    if (!sep23 && equ_zero(r1)) {
        reserved = 1;
        return INTER_T1;
    }
    if (equ_zero(r2) && equ_zero(r3)) return INTER_OVERLAP;
    if (!sep01 && equ_zero(r2)) {
        reserved = 0;
        return INTER_T2;
    }
    if (!sep01 && equ_zero(r3)) {
        reserved = 1;
        return INTER_T2;
    }
    if (sep01 || sep23) return INTER_NO;
    return INTER_X;
}

__device__ __forceinline__ int seg_exit_border(D3 p0, D3 p1, const GridView& g, int cid, int in, int& intertype,
                                               int& info)
{
    const int bs = g.C[cid].bstart, be = bs + g.C[cid].bnum;
    for (int i = bs; i < be; i++) {
        if (i == in) continue;
        int temp = 0;
        const Border bi = g.B[i];
        int inter = edge_border_inter(p0, p1, g.V[bi.v[0]], g.V[bi.v[1]], temp);
        if (inter == INTER_X) {
            intertype = INTER_X;
            return i;
        }
        if (inter == INTER_T1) {
            intertype = INTER_T1;
            if (temp == 0) {
                info = 0;
                return i;
            }
            info = 1;
            return -1;
        }
        if (inter == INTER_T2) {
            if (in != -1) {
                const int vt = bi.v[temp];
                if (vt == g.B[in].v[0] || vt == g.B[in].v[1]) continue;
            }
            intertype = INTER_T2;
            info = temp;
            return i;
        }
        if (inter == INTER_OVERLAP) {
            intertype = INTER_OVERLAP;
            return i;
        }
    }
    return -1;
}

enum WalkMode { WALK_MARK = 0, WALK_COUNT = 1, WALK_WRITE = 2 };

// Finds the cell of `p` at level 0 (linear over cells 0..n0-1) or among the
// center subcell and border subcells of `prev` (the cell at the level above).
__device__ __forceinline__ int locate_start(D3 p, int level, int n0, int prev, const GridView& g)
{
    int cur = -1;
    if (level == 0) {
        for (int i = 0; i < n0; i++) {
            cur = inside_cell(p, i, g);
            if (cur != -1) break;
        }
        return cur;
    }
    if (prev < 0 || prev >= g.nc) return -2;
    cur = inside_cell(p, g.C[prev].subcell, g);
    if (cur == -1) {
        const int bs = g.C[prev].bstart, bn = g.C[prev].bnum;
        for (int i = 0; i < bn; i++) {
            cur = g.B[bs + i].subcell;
            if (cur == -1) continue;
            cur = inside_cell(p, cur, g);
            if (cur != -1) break;
        }
    }
    return cur;
}

// Walks edge p0->p1 from `cur` through the cell graph.  Returns the number of
// cells visited; visits are reported through `visit(cell, k)`.
template <int MODE, class Visit>
__device__ __forceinline__ int walk_edge(D3 p0, D3 p1, int cur, const GridView& g, DeviceErrors* err, Visit visit)
{
    int in = -1;
    int steps = 0;
    int seen_cur = cur, seen_in = in, window = 1, since = 0;  // Brent's cycle test
    while (true) {
        if (steps >= g.walk_limit || (steps > 0 && cur == seen_cur && in == seen_in)) {
            atomicAdd(&err->walk_step_limit, 1);
            return steps;
        }
        if (++since == window) {
            seen_cur = cur;
            seen_in = in;
            window <<= 1;
            since = 0;
        }
        visit(cur, steps);
        steps++;
        int intertype = 0, info = 0;
        const int out = seg_exit_border(p0, p1, g, cur, in, intertype, info);
        if (out == -1) break;
        if (intertype == INTER_X || intertype == INTER_T1) {
            in = g.B[out].partner;
            if (in < 0 || in >= g.nb) {
                atomicAdd(&err->walk_bad_index, 1);
                return steps;
            }
            cur = g.B[in].parent;
        } else if (intertype == INTER_T2) {
            D3 curpoint = g.V[g.B[out].v[info]];
            D3 e = normalize(p1 - p0);
            curpoint = curpoint + e * TRAVEL_EPSILON;
            const int u = g.C[cur].bnum;
            const int op = g.B[out].partner;
            if (op != -1) {
                int ret = inside_cell(curpoint, g.B[op].parent, g);
                if (ret != -1) {
                    cur = ret;
                    in = op;
                    continue;
                }
            }
            const int oid = g.B[out].id;
            const int other = g.C[cur].bstart + (info == 0 ? (oid + u - 1) % u : (oid + 1) % u);
            const int pp = g.B[other].partner;
            if (pp != -1) {
                int ret = inside_cell(curpoint, g.B[pp].parent, g);
                if (ret != -1) {
                    cur = ret;
                    in = pp;
                    continue;
                }
                return steps;
            }
            return steps;
        } else if (intertype == INTER_OVERLAP) {
            D3 e0 = normalize(p1 - p0);
            D3 e1 = normalize(g.V[g.B[out].v[1]] - g.V[g.B[out].v[0]]);
            double temp = dot(e0, e1);
            const int u = g.C[cur].bnum;
            if (MODE == WALK_MARK) {
                // source/GPISPAHHG.cu:1277-1285 computes `in` from the cell it
                // has just moved to; kept as written.
                const int bs0 = g.C[cur].bstart;
                const int step = temp > 0 ? 1 : u - 1;
                const int target = bs0 + (out - bs0 + step) % u;
                const int tp = g.B[target].partner;
                if (tp < 0 || tp >= g.nb) {
                    atomicAdd(&err->walk_bad_index, 1);
                    return steps;
                }
                cur = g.B[tp].parent;
                const int bs1 = g.C[cur].bstart;
                const int idx = bs1 + (out - bs1 + step) % u;
                if (idx < 0 || idx >= g.nb) {
                    atomicAdd(&err->walk_bad_index, 1);
                    return steps;
                }
                in = g.B[idx].partner;
            } else {
                const int target = g.C[cur].bstart + (temp > 0 ? (g.B[out].id + 1) % u : (g.B[out].id + u - 1) % u);
                const int tp = g.B[target].partner;
                if (tp < 0 || tp >= g.nb) {
                    atomicAdd(&err->walk_bad_index, 1);
                    return steps;
                }
                cur = g.B[tp].parent;
                in = tp;
            }
        }
    }
    return steps;
}

}  // namespace gahhg
