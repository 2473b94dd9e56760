// classify.cu - IN/OUT labels for the cells of the hexagon hierarchy.
//
// Reference semantics (GAHHG::classifyBottomGrid source/GPISPAHHG.cu:1787-1817,
// GPISP::classifyAHHG :2018-2059, kernels :1046-1124, :1292-1419, predicates
// device_getCPProp :61-171 and dev_isInterSeg :174-205), FP64 with the same
// operation order.
//
// Three of the reference kernels (setBottomDECell, setIECell, setTopECell)
// read neighbour types that other threads of the same launch are writing, so
// the reference's result depends on thread scheduling.  This file computes
// the result of one fixed schedule - every thread of a launch run to
// completion in increasing thread index - which is also what the reference
// produces when it is run serially.  On the GPU that schedule is reached by a
// fixpoint: round k recomputes every cell from the types of lower-indexed
// cells as of round k-1 and of higher-indexed cells as of the launch start;
// the fixpoint is unique and equals the serial result.  setTopECell (42 cells)
// runs serially in one thread.
#include <cstdio>
#include <cfloat>

#include "gahhg_internal.h"
#include "walk.cuh"

namespace gahhg {

namespace {

constexpr int TPB = 256;
inline int blocks_for(long long n) { return (int)((n + TPB - 1) / TPB > 0 ? (n + TPB - 1) / TPB : 1); }
constexpr int GS_MAX_ROUNDS = 1 << 14;

struct ClassView {
    const D3* pv;
    const int* pe;
    const D3* V;
    const Border* B;
    Cell* C;
    const int* refs;
};

__device__ __forceinline__ D3 cell_center(const ClassView& g, int cell)
{
    const int bs = g.C[cell].bstart, bn = g.C[cell].bnum;
    D3 c = d3(0.0, 0.0, 0.0);
    for (int i = 0; i < bn; i++) c = c + g.V[g.B[bs + i].v[0]];
    c = c / (double)bn;
    return normalize(c);
}

// device_getCPProp (source/GPISPAHHG.cu:61-171): side of the nearest edge.
__device__ int cp_prop(const ClassView& g, int cell, D3 center)
{
    double mindist = FLT_MAX;
    const int rs = g.C[cell].rstart, rn = g.C[cell].rnum;
    int ne = g.refs[rs];
    D3 ne_normal = d3(0.0, 0.0, 0.0);
    int nv_index = -1;
    for (int i = 0; i < rn; i++) {
        const int se = g.refs[rs + i];
        const D3 v0 = g.pv[g.pe[2 * se]], v1 = g.pv[g.pe[2 * se + 1]];
        double curdist = FLT_MAX;
        D3 n0 = normalize(cross(v0, v1 - v0));
        D3 n1 = normalize(cross(center, n0));
        D3 inter = normalize(cross(n0, n1));
        double temp = dot(inter, v0);
        if (less_zero(temp)) inter = -inter;
        D3 t0 = normalize(v0 - inter);
        D3 t1 = normalize(v1 - inter);
        double temp3 = dot(t0, t1);
        int cur_nv = -1;
        if (less_zero(temp3)) {
            curdist = squarelen(inter - center);
            cur_nv = -1;
        } else {
            curdist = squarelen(center - v0);
            double vdist = squarelen(center - v1);
            if (vdist < curdist) {
                curdist = vdist;
                cur_nv = g.pe[2 * se + 1];
            } else {
                cur_nv = g.pe[2 * se];
            }
        }
        if (nv_index != -1 && nv_index == cur_nv) {
            double a = dot(ne_normal, center);
            double b = dot(n0, center);
            if ((less_equ_zero(a) && gre_equ_zero(b)) || (gre_equ_zero(a) && less_equ_zero(b))) {
                int other = (g.pe[2 * ne] == nv_index) ? g.pe[2 * ne + 1] : g.pe[2 * ne];
                D3 a0 = g.pv[other] - g.pv[nv_index];
                other = (g.pe[2 * se] == nv_index) ? g.pe[2 * se + 1] : g.pe[2 * se];
                D3 a1 = g.pv[other] - g.pv[nv_index];
                D3 bb = center - g.pv[nv_index];
                a0 = normalize(a0);
                a1 = normalize(a1);
                a = dot(a0, bb);
                b = dot(a1, bb);
                if (b > a) {
                    mindist = curdist;
                    ne = se;
                    ne_normal = n0;
                    nv_index = cur_nv;
                    continue;
                }
            }
        }
        if (curdist < mindist) {
            mindist = curdist;
            ne = se;
            ne_normal = n0;
            nv_index = cur_nv;
        }
    }
    double temp = dot(center, ne_normal);
    return gre_zero(temp) ? CELL_IN : CELL_OUT;
}

// dev_isInterSeg (source/GPISPAHHG.cu:174-205)
__device__ __forceinline__ bool inter_seg(D3 v0, D3 v1, D3 p0, D3 p1)
{
    D3 n0 = normalize(cross(v0, v1 - v0));
    double r0 = dot(n0, p0), r1 = dot(n0, p1);
    if ((less_zero(r0) && less_zero(r1)) || (gre_zero(r0) && gre_zero(r1))) return false;
    D3 n1 = normalize(cross(p0, p1 - p0));
    r0 = dot(n1, v0);
    r1 = dot(n1, v1);
    if ((less_zero(r0) && less_zero(r1)) || (gre_zero(r0) && gre_zero(r1))) return false;
    return true;
}

// parity of the polygon edges of `cell` crossing arc(center(cell), midpoint of border e)
__device__ int crossing_parity(const ClassView& g, int cell, int e)
{
    D3 mid = normalize((g.V[g.B[e].v[0]] + g.V[g.B[e].v[1]]) * 0.5);
    D3 center = cell_center(g, cell);
    int count = 0;
    const int rs = g.C[cell].rstart, rn = g.C[cell].rnum;
    for (int i = 0; i < rn; i++) {
        const int se = g.refs[rs + i];
        if (inter_seg(g.pv[g.pe[2 * se]], g.pv[g.pe[2 * se + 1]], center, mid)) count++;
    }
    return count & 1;
}

// kernel_Classify_setBottomNECell (:1046-1071)
__global__ void k_bottom_ne(ClassView g, int cs, int cn)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cn) return;
    const int cell = cs + t;
    if (g.C[cell].rnum == 0) return;
    g.C[cell].type = cp_prop(g, cell, cell_center(g, cell));
}

__global__ void k_gather_types(const Cell* C, int cs, int cn, int* a, int* b)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cn) return;
    a[t] = b[t] = C[cs + t].type;
}

__global__ void k_scatter_types(Cell* C, int cs, int cn, const int* a)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < cn) C[cs + t].type = a[t];
}

// Type of cell u as thread t of a serial run would see it.
__device__ __forceinline__ int seen_type(const Cell* C, int u, int t, int cs, int cn, const int* old, const int* cur)
{
    const int k = u - cs;
    if (k < 0 || k >= cn) return C[u].type;
    return k < t ? cur[k] : old[k];
}

// kernel_Classify_setBottomDECell (:1074-1124), one fixpoint round.
__global__ void k_bottom_de_round(ClassView g, int cs, int cn, const int* old, const int* cur, int* next,
                                  int* changed)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cn) return;
    int ty = old[t];
    if (ty == CELL_UNDEFINED) {
        const int bs = g.C[cs + t].bstart, bn = g.C[cs + t].bnum;
        for (int i = 0; i < bn; i++) {
            const int pe = g.B[bs + i].partner;
            if (pe == -1) continue;
            const int u = g.B[pe].parent;
            const int tu = seen_type(g.C, u, t, cs, cn, old, cur);
            if (tu == CELL_UNDEFINED) continue;
            ty = crossing_parity(g, u, pe) == 0 ? tu : 3 - tu;
        }
    }
    next[t] = ty;
    if (ty != cur[t]) *changed = 1;
}

// kernel_Classify_setIECell (:1366-1392), one fixpoint round.
__global__ void k_ie_round(ClassView g, int cs, int cn, const int* old, const int* cur, int* next, int* changed)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cn) return;
    int ty = old[t];
    const Cell c = g.C[cs + t];
    if (ty == CELL_UNDEFINED && c.subcell == -1) {
        for (int i = 0; i < c.bnum; i++) {
            const int pe = g.B[c.bstart + i].partner;
            if (pe == -1) continue;
            const int u = g.B[pe].parent;
            const int tu = seen_type(g.C, u, t, cs, cn, old, cur);
            if (g.C[u].rnum == 0 && tu != CELL_UNDEFINED) {
                ty = tu;
                break;
            }
        }
    }
    next[t] = ty;
    if (ty != cur[t]) *changed = 1;
}

// kernel_Classify_setDECell (:1292-1363): reads only deeper, final cells.
__global__ void k_level_de(ClassView g, int cs, int cn)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cn) return;
    const int cell = cs + t;
    const Cell c = g.C[cell];
    if (!(c.rnum == 0 && c.type == CELL_UNDEFINED)) return;
    int pedge = -1, pcell = -1;
    for (int i = 0; i < c.bnum; i++) {
        pedge = g.B[c.bstart + i].partner;
        if (pedge != -1 && g.C[g.B[pedge].parent].subcell != -1) {
            pcell = g.B[pedge].parent;
            break;
        }
    }
    if (pcell == -1) return;
    int target = g.B[pedge].subcell;
    if (target < 0) return;  // the reference would read cell -1 here
    for (int guard = 0; g.C[target].subcell != -1 && guard < 64; guard++) target = g.C[target].subcell;
    if (g.C[target].rnum == 0) {
        g.C[cell].type = g.C[target].type;
        return;
    }
    const int tt = g.C[target].type;
    g.C[cell].type = crossing_parity(g, target, pedge) == 0 ? tt : 3 - tt;
}

// kernel_Classify_setTopECell (:1395-1419) in serial thread order.
__global__ void k_top_serial(const Border* B, Cell* C, int cn)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int t = 0; t < cn; t++) {
        for (int j = 0; j < 3; j++) {
            if (C[t].rnum == 0 && C[t].type == CELL_UNDEFINED) {
                for (int i = 0; i < C[t].bnum; i++) {
                    const int pe = B[C[t].bstart + i].partner;
                    if (pe != -1 && C[B[pe].parent].type != CELL_UNDEFINED) {
                        C[t].type = C[B[pe].parent].type;
                        break;
                    }
                }
            }
        }
    }
}

// Serial fallback for a fixpoint that did not settle within GS_MAX_ROUNDS.
__global__ void k_serial_round(ClassView g, int cs, int cn, int* old, int* cur, int kind)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int t = 0; t < cn; t++) {
        int ty = old[t];
        const Cell c = g.C[cs + t];
        if (kind == 0) {
            if (ty == CELL_UNDEFINED) {
                for (int i = 0; i < c.bnum; i++) {
                    const int pe = g.B[c.bstart + i].partner;
                    if (pe == -1) continue;
                    const int u = g.B[pe].parent;
                    const int tu = seen_type(g.C, u, t, cs, cn, old, cur);
                    if (tu == CELL_UNDEFINED) continue;
                    ty = crossing_parity(g, u, pe) == 0 ? tu : 3 - tu;
                }
            }
        } else if (ty == CELL_UNDEFINED && c.subcell == -1) {
            for (int i = 0; i < c.bnum; i++) {
                const int pe = g.B[c.bstart + i].partner;
                if (pe == -1) continue;
                const int u = g.B[pe].parent;
                const int tu = seen_type(g.C, u, t, cs, cn, old, cur);
                if (g.C[u].rnum == 0 && tu != CELL_UNDEFINED) {
                    ty = tu;
                    break;
                }
            }
        }
        cur[t] = ty;
    }
}

}  // namespace

// Runs one racy reference kernel (kind 0 = setBottomDECell, 1 = setIECell)
// over cells [cs, cs+cn) with serial-schedule semantics.
static gahhg_status serial_schedule(Grid* g, const ClassView& v, int cs, int cn, int kind)
{
    if (cn <= 0) return GAHHG_OK;
    cudaStream_t s = g->stream;
    GAHHG_TRY(g->type_old.reserve(cn, s, false));
    GAHHG_TRY(g->type_cur.reserve(cn, s, false));
    GAHHG_TRY(g->type_next.reserve(cn, s, false));
    k_gather_types<<<blocks_for(cn), TPB, 0, s>>>(v.C, cs, cn, g->type_old.ptr, g->type_cur.ptr);
    int* d_changed = g->d_counts + 32;
    int* cur = g->type_cur.ptr;
    int* next = g->type_next.ptr;
    bool settled = false;
    for (int round = 0; round < GS_MAX_ROUNDS;) {
        // a batch of rounds between host checks; extra rounds at the fixpoint change nothing
        const int batch = round < 8 ? 2 : 8;
        GAHHG_CUDA_TRY(cudaMemsetAsync(d_changed, 0, sizeof(int), s));
        for (int k = 0; k < batch; k++, round++) {
            if (k == batch - 1) GAHHG_CUDA_TRY(cudaMemsetAsync(d_changed, 0, sizeof(int), s));
            if (kind == 0)
                k_bottom_de_round<<<blocks_for(cn), TPB, 0, s>>>(v, cs, cn, g->type_old.ptr, cur, next, d_changed);
            else
                k_ie_round<<<blocks_for(cn), TPB, 0, s>>>(v, cs, cn, g->type_old.ptr, cur, next, d_changed);
            std::swap(cur, next);
        }
        GAHHG_CUDA_TRY(cudaGetLastError());
        int changed = 0;
        GAHHG_CUDA_TRY(cudaMemcpyAsync(&changed, d_changed, sizeof(int), cudaMemcpyDeviceToHost, s));
        GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
        if (!changed) {
            settled = true;
            break;
        }
    }
    if (!settled) k_serial_round<<<1, 1, 0, s>>>(v, cs, cn, g->type_old.ptr, cur, kind);
    k_scatter_types<<<blocks_for(cn), TPB, 0, s>>>(v.C, cs, cn, cur);
    GAHHG_CUDA_TRY(cudaGetLastError());
    return GAHHG_OK;
}

gahhg_status grid_classify(Grid* g)
{
    cudaStream_t s = g->stream;
    ClassView v;
    v.pv = g->poly->d_pv;
    v.pe = g->poly->d_pe;
    v.V = g->V.ptr;
    v.B = g->B.ptr;
    v.C = g->C.ptr;
    v.refs = g->refs.ptr;
    const double t0 = now_seconds();
    const Level& bot = g->levels[g->gnum - 1];
    if (g->opts.verbose) printf("Classify level %d cells.\n", g->gnum - 1);
    k_bottom_ne<<<blocks_for(bot.cnum), TPB, 0, s>>>(v, bot.cstart, bot.cnum);
    GAHHG_TRY(serial_schedule(g, v, bot.cstart, bot.cnum, 0));
    GAHHG_TRY(serial_schedule(g, v, bot.cstart, bot.cnum, 1));
    for (int i = g->gnum - 2; i >= 0; i--) {
        if (g->opts.verbose) printf("Classify level %d cells.\n", i);
        const Level& L = g->levels[i];
        k_level_de<<<blocks_for(L.cnum), TPB, 0, s>>>(v, L.cstart, L.cnum);
        GAHHG_TRY(serial_schedule(g, v, L.cstart, L.cnum, 1));
    }
    k_top_serial<<<1, 1, 0, s>>>(g->B.ptr, g->C.ptr, g->levels[0].cnum);
    GAHHG_CUDA_TRY(cudaGetLastError());
    GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
    g->stats.classify_s = now_seconds() - t0;
    g->stats.pre_s = g->stats.create_s + g->stats.classify_s;
    GAHHG_TRY(check_device_errors(g, "classify"));
    g->classified = true;
    return GAHHG_OK;
}

}  // namespace gahhg
