// build.cu - level-synchronous construction of the hexagon hierarchy on the GPU.
//
// Reference semantics (GAHHG::divGrid source/GPISPAHHG.cu:1558-1697,
// GAHHG::dispatchSELast :1700-1784, GPISP::createAHHG :1976-2015): the same
// cells, vertices, borders and edge lists, numbered the same way, so the
// grid arrays equal the reference's bit for bit.  What changes is the
// execution: counts come from a single-pass look-back scan whose totals land
// in one small device header, so each level costs one host round trip
// instead of seven; buffers are reserved from upper bounds known at that
// round trip; the bottom-level cell->edge lists are ordered by edge (the
// reference's atomic scatter leaves the order to the scheduler, which the
// reference itself depends on only in nearest-edge ties).
#include <cstdio>
#include <cstring>

#include "walk.cuh"

namespace gahhg {

gahhg_status scan_state_reserve(void** state, size_t max_n);
void scan_state_destroy(void* state);

namespace {

constexpr int TPB = 256;
inline int blocks_for(long long n) { return (int)((n + TPB - 1) / TPB > 0 ? (n + TPB - 1) / TPB : 1); }

// Device header of counts read back once per level.
enum {
    HC_SUM_A = 0,   // new center-subcell vertices/borders
    HC_SUM_B,       // marked cells (new center subcells) = gamma numerator
    HC_SUM_A2,      // border-subcell borders
    HC_SUM_B2,      // border subcells
    HC_REFS,        // bottom-level refs
    HC_NUM
};

__global__ void k_zero_ref_count(Cell* C, Border* B, int cstart, int cnum)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cnum) return;
    Cell& c = C[cstart + t];
    c.rnum = 0;
    if (cstart == 0) {
        c.rstart = -1;
        c.subcell = -1;
        c.upcell = -1;
        c.type = CELL_UNDEFINED;
        for (int i = 0; i < c.bnum; i++) B[c.bstart + i].subcell = -1;
    }
}

__global__ void k_mark(const D3* __restrict__ pv, const int* __restrict__ pe, int pv_num, GridView g, int level,
                       int* buf_prev, int* buf_cur, DeviceErrors* err)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= pv_num) return;
    const D3 p0 = pv[pe[2 * t]], p1 = pv[pe[2 * t + 1]];
    buf_prev[t] = buf_cur[t];
    int cur = locate_start(p0, level, 42, buf_cur[t], g);
    if (cur == -2) {
        atomicAdd(&err->walk_bad_index, 1);
        return;
    }
    if (cur == -1) return;
    buf_cur[t] = cur;
    Cell* C = g.C;
    walk_edge<WALK_MARK>(p0, p1, cur, g, err, [&](int c, int) { C[c].rnum = 999; });
}

__global__ void k_center_offsets(const Cell* C, int cstart, int cnum, int* a, int* b)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cnum) return;
    const Cell c = C[cstart + t];
    a[t] = c.rnum == 0 ? 0 : c.bnum;
    b[t] = c.rnum == 0 ? 0 : 1;
}

__global__ void k_create_center(D3* V, int vs, Border* B, int bs, Cell* C, int cstart, int cnum,
                                const int* off_a, const int* off_b)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cnum) return;
    const Cell pc = C[cstart + t];
    if (pc.rnum == 0) return;
    D3 center = d3(0.0, 0.0, 0.0);
    if (pc.bnum == 4) {
        center = (V[B[pc.bstart].v[0]] + V[B[pc.bstart].v[1]]) * 0.5;
    } else {
        for (int i = 0; i < pc.bnum; i++) center = center + V[B[pc.bstart + i].v[0]];
        center = center / (double)pc.bnum;
    }
    center = normalize(center);
    const int v0 = vs + off_a[t], b0 = bs + off_a[t], cnew = cstart + cnum + off_b[t];
    for (int i = 0; i < pc.bnum; i++) V[v0 + i] = normalize((V[B[pc.bstart + i].v[0]] + center) * 0.5);
    for (int i = 0; i < pc.bnum; i++) {
        Border nb;
        nb.id = i;
        nb.parent = cnew;
        nb.partner = -1;
        nb.subcell = -1;
        nb.v[0] = v0 + i;
        nb.v[1] = v0 + (i + 1) % pc.bnum;
        D3 n = edge_normal(V[nb.v[0]], V[nb.v[1]]);
        nb.n[0] = n.x;
        nb.n[1] = n.y;
        nb.n[2] = n.z;
        B[b0 + i] = nb;
    }
    Cell nc;
    nc.bstart = b0;
    nc.bnum = pc.bnum;
    nc.rstart = -1;
    nc.rnum = -1;
    nc.upcell = cstart + t;
    nc.subcell = -1;
    nc.type = CELL_UNDEFINED;
    C[cnew] = nc;
    C[cstart + t].subcell = cnew;
}

// Which border subcell (hex shared with a refined neighbour, or quad toward
// an unrefined one) the parent edge under new border `nb` gets
// (source/GPISPAHHG.cu:473-509).  0 = none, 6 = hex, 4 = quad.
__device__ __forceinline__ int border_sc_kind(const Border* B, const Cell* C, const Border& nb, int& upedge_idx)
{
    const Cell upcell = C[C[nb.parent].upcell];
    upedge_idx = upcell.bstart + nb.id;
    const Border ue = B[upedge_idx];
    if (upcell.bnum == 4 && nb.id == 0) return 0;
    if (ue.partner != -1 && C[B[ue.partner].parent].subcell != -1 && ue.parent < B[ue.partner].parent) return 6;
    if (ue.partner == -1 || (ue.partner != -1 && C[B[ue.partner].parent].subcell == -1)) return 4;
    return 0;
}

__global__ void k_border_sc_offsets(const Border* B, const Cell* C, int bs, int bnum, int* a, int* b)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= bnum) return;
    int ue;
    int k = border_sc_kind(B, C, B[bs + t], ue);
    a[t] = k;
    b[t] = k ? 1 : 0;
}

__global__ void k_create_border_sc(const D3* V, Border* B, int bs, int bnum, Cell* C, int cs, int cnum,
                                   const int* off_a, const int* off_b)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= bnum) return;
    const Border nb = B[bs + t];
    int ue;
    const int kind = border_sc_kind(B, C, nb, ue);
    if (!kind) return;
    const Border up = B[ue];
    const int eoff = bs + bnum + off_a[t];
    const int coff = cs + cnum + off_b[t];
    int vv[6];
    if (kind == 6) {
        const Cell psc = C[C[B[up.partner].parent].subcell];
        const Border pse = B[psc.bstart + B[up.partner].id];
        vv[0] = up.v[0];
        vv[1] = pse.v[1];
        vv[2] = pse.v[0];
        vv[3] = up.v[1];
        vv[4] = nb.v[1];
        vv[5] = nb.v[0];
    } else {
        vv[0] = up.v[0];
        vv[1] = up.v[1];
        vv[2] = nb.v[1];
        vv[3] = nb.v[0];
    }
    for (int i = 0; i < kind; i++) {
        Border sb;
        sb.id = i;
        sb.v[0] = vv[i];
        sb.v[1] = vv[(i + 1) % kind];
        sb.parent = coff;
        sb.partner = -1;
        D3 n = edge_normal(V[sb.v[0]], V[sb.v[1]]);
        sb.n[0] = n.x;
        sb.n[1] = n.y;
        sb.n[2] = n.z;
        sb.subcell = -1;
        B[eoff + i] = sb;
    }
    Cell c;
    c.bnum = kind;
    c.bstart = eoff;
    c.rstart = -1;
    c.rnum = -1;
    c.subcell = -1;
    c.upcell = up.parent;
    c.type = CELL_UNDEFINED;
    C[coff] = c;
    B[ue].subcell = coff;
    if (kind == 6) B[up.partner].subcell = coff;
}

// device_setBorderPartner (source/GPISPAHHG.cu:42-58)
__device__ __forceinline__ void set_border_partner(const Cell* C, Border* B, int cell, int e)
{
    const int bs = C[cell].bstart, bn = C[cell].bnum;
    const int e0 = B[e].v[0], e1 = B[e].v[1];
    for (int i = 0; i < bn; i++) {
        const int j = bs + i;
        if (e0 == B[j].v[1] && e1 == B[j].v[0] && e < j) {
            B[e].partner = j;
            B[j].partner = e;
        }
    }
}

// kernel_DivGrid_setSCPartner (source/GPISPAHHG.cu:610-682)
__global__ void k_set_sc_partner(Border* B, const Cell* C, int cs, int cnum)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cnum) return;
    const int cell = cs + t;
    const Cell cur = C[cell];
    // device_getUpEdgeForSubcell (:27-39)
    int upedge = -1;
    {
        const Cell upc = C[cur.upcell];
        for (int i = 0; i < upc.bnum; i++)
            if (B[upc.bstart + i].subcell == cell) {
                upedge = upc.bstart + i;
                break;
            }
    }
    if (upedge == -1) return;
    const Cell upc = C[cur.upcell];
    const int uid = B[upedge].id;
    auto link_or_clear = [&](int tempedge, int mine) {
        if (B[tempedge].subcell != -1)
            set_border_partner(C, B, B[tempedge].subcell, mine);
        else
            B[mine].partner = -1;
    };
    if (cur.bnum == 6) {
        const int pedge = B[upedge].partner;
        const int pcell = B[pedge].parent;
        const int u = C[pcell].bnum;
        const int pid = B[pedge].id;
        link_or_clear(C[pcell].bstart + (pid + 1) % u, cur.bstart);
        int te = C[C[pcell].subcell].bstart + pid;
        B[cur.bstart + 1].partner = te;
        B[te].partner = cur.bstart + 1;
        link_or_clear(C[pcell].bstart + (pid + u - 1) % u, cur.bstart + 2);
        link_or_clear(upc.bstart + (uid + 1) % upc.bnum, cur.bstart + 3);
        te = C[upc.subcell].bstart + uid;
        B[cur.bstart + 4].partner = te;
        B[te].partner = cur.bstart + 4;
        link_or_clear(upc.bstart + (uid + upc.bnum - 1) % upc.bnum, cur.bstart + 5);
    } else if (cur.bnum == 4) {
        link_or_clear(upc.bstart + (uid + 1) % upc.bnum, cur.bstart + 1);
        int te = C[upc.subcell].bstart + uid;
        B[cur.bstart + 2].partner = te;
        B[te].partner = cur.bstart + 2;
        link_or_clear(upc.bstart + (uid + upc.bnum - 1) % upc.bnum, cur.bstart + 3);
    }
}

// kernel_calcRefNum / kernel_writeRef (source/GPISPAHHG.cu:685-955)
template <int MODE>
__global__ void k_edge_refs(const D3* __restrict__ pv, const int* __restrict__ pe, int pv_num, GridView g,
                            int level, int ncell_level0, int* buf, int* cnt, const int* off, int* ref_cell,
                            DeviceErrors* err)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= pv_num) return;
    const D3 p0 = pv[pe[2 * t]], p1 = pv[pe[2 * t + 1]];
    int cur = locate_start(p0, level, ncell_level0, level == 0 ? -1 : buf[t], g);
    if (cur == -2) {
        atomicAdd(&err->walk_bad_index, 1);
        if (MODE == WALK_COUNT) cnt[t] = 0;
        return;
    }
    if (cur == -1) {
        if (MODE == WALK_COUNT) cnt[t] = 0;
        return;
    }
    if (MODE == WALK_WRITE && level != 0) buf[t] = cur;
    if (MODE == WALK_COUNT) {
        cnt[t] = walk_edge<WALK_COUNT>(p0, p1, cur, g, err, [](int, int) {});
    } else {
        int* dst = ref_cell + off[t];
        const int limit = cnt[t];
        walk_edge<WALK_WRITE>(p0, p1, cur, g, err, [&](int c, int k) {
            if (k < limit) dst[k] = c;
        });
    }
}

// kernel_EC2CS_setEFlag (:971-981): head flag at each edge's first ref.
// Edges without refs share their offset with the next edge, so the flag
// count (and the edge index recovered from it) falls behind, exactly as in
// the reference.
__global__ void k_edge_flags(const int* off, int pv_num, int* flag, int nref)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 || i >= pv_num) return;
    int o = off[i];
    if (o < nref) flag[o] = 1;
}

__global__ void k_add(const int* a, int* b, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] += a[i];
}

__global__ void k_count_per_cell(const int* ref_cell, int nref, int cstart, int cnum, int* cell_cnt,
                                 DeviceErrors* err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nref) return;
    int c = ref_cell[i] - cstart;
    if (c < 0 || c >= cnum) {
        atomicAdd(&err->walk_bad_index, 1);
        return;
    }
    atomicAdd(&cell_cnt[c], 1);
}

__global__ void k_scatter_refs(const int* ref_cell, const int* ref_edge, int nref, int cstart, int cnum,
                               int* cursor, int* refs_out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nref) return;
    int c = ref_cell[i] - cstart;
    if (c < 0 || c >= cnum) return;
    int pos = atomicAdd(&cursor[c], 1);
    refs_out[pos] = ref_edge[i];
}

// Orders each cell's edge list ascending, which is the order a serial run of
// the reference's scatter produces (refs are laid out edge after edge).
__global__ void k_sort_cell_refs(Cell* C, int cstart, int cnum, const int* cell_cnt, const int* cell_off,
                                 int* refs)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cnum) return;
    const int n = cell_cnt[t], o = cell_off[t];
    for (int i = 1; i < n; i++) {
        int x = refs[o + i];
        int j = i - 1;
        while (j >= 0 && refs[o + j] > x) {
            refs[o + j + 1] = refs[o + j];
            j--;
        }
        refs[o + j + 1] = x;
    }
    C[cstart + t].rnum = n;
    C[cstart + t].rstart = o;
}

}  // namespace

// -------------------------------------------------------------------- host --



gahhg_status check_device_errors(Grid* g, const char* phase)
{
    DeviceErrors e;
    GAHHG_CUDA_TRY(cudaMemcpyAsync(&e, g->d_err, sizeof(e), cudaMemcpyDeviceToHost, g->stream));
    GAHHG_CUDA_TRY(cudaStreamSynchronize(g->stream));
    // A walk that reaches the step limit is a walk the reference would never
    // finish (its loops are unbounded); the build completes and reports it.
    g->stats.walk_limit_hits = e.walk_step_limit;
    // a scan whose look-back ran out of time summed the late tile's inputs
    // itself: its result is exact, the event is only counted
    g->stats.scan_fallbacks = e.scan_lookback_timeout;
    if (e.classify_no_converge || e.lattice_overflow || e.other) {
        set_error("%s: device reported walk_step_limit=%d scan_timeout=%d classify_no_converge=%d "
                  "lattice_overflow=%d other=%d",
                  phase, e.walk_step_limit, e.scan_lookback_timeout, e.classify_no_converge, e.lattice_overflow,
                  e.other);
        return GAHHG_ERR_DEVICE;
    }
    return GAHHG_OK;
}

static GridView view(Grid* g)
{
    const Level& L = g->levels[g->gnum - 1];
    GridView v;
    v.V = g->V.ptr;
    v.B = g->B.ptr;
    v.C = g->C.ptr;
    v.nb = L.bstart + L.bnum;
    v.nc = L.cstart + L.cnum;
    v.walk_limit = (int)knob(GAHHG_KNOB_WALK_STEP_LIMIT);
    return v;
}

static gahhg_status read_counts(Grid* g)
{
    GAHHG_CUDA_TRY(cudaMemcpyAsync(g->h_counts, g->d_counts, HC_NUM * sizeof(int), cudaMemcpyDeviceToHost, g->stream));
    GAHHG_CUDA_TRY(cudaStreamSynchronize(g->stream));
    return GAHHG_OK;
}

// One refinement step (GAHHG::divGrid).  Returns GAHHG_OK and sets *more to
// false when the auto-depth rule stops the refinement at this level.
static gahhg_status div_grid(Grid* g, int L, bool* more)
{
    cudaStream_t s = g->stream;
    const Polygon* P = g->poly;
    if (g->opts.verbose) printf("Subdivide level %d on GPU.\n", L);
    Level lv = g->levels[L];

    k_zero_ref_count<<<blocks_for(lv.cnum), TPB, 0, s>>>(g->C.ptr, g->B.ptr, lv.cstart, lv.cnum);
    GridView gv;
    gv.V = g->V.ptr;
    gv.B = g->B.ptr;
    gv.C = g->C.ptr;
    gv.nb = lv.bstart + lv.bnum;
    gv.nc = lv.cstart + lv.cnum;
    gv.walk_limit = (int)knob(GAHHG_KNOB_WALK_STEP_LIMIT);
    k_mark<<<blocks_for(P->pv_num), TPB, 0, s>>>(P->d_pv, P->d_pe, P->pv_num, gv, L, g->edge_prev.ptr,
                                                 g->edge_cur.ptr, g->d_err);
    GAHHG_TRY(g->cell_a.reserve(lv.cnum, s, false));
    GAHHG_TRY(g->cell_b.reserve(lv.cnum, s, false));
    GAHHG_TRY(g->off_a.reserve(lv.cnum, s, false));
    GAHHG_TRY(g->off_b.reserve(lv.cnum, s, false));
    k_center_offsets<<<blocks_for(lv.cnum), TPB, 0, s>>>(g->C.ptr, lv.cstart, lv.cnum, g->cell_a.ptr, g->cell_b.ptr);
    GAHHG_TRY(scan_state_reserve(&g->scan_state, lv.cnum));
    GAHHG_TRY(scan_exclusive(g->cell_a.ptr, g->off_a.ptr, lv.cnum, g->d_counts + HC_SUM_A, g->scan_state, g->d_err, s));
    GAHHG_TRY(scan_exclusive(g->cell_b.ptr, g->off_b.ptr, lv.cnum, g->d_counts + HC_SUM_B, g->scan_state, g->d_err, s));
    GAHHG_CUDA_TRY(cudaGetLastError());
    GAHHG_TRY(read_counts(g));
    const int sumA = g->h_counts[HC_SUM_A], sumB = g->h_counts[HC_SUM_B];

    if (g->opts.auto_depth) {
        // source/GPISPAHHG.cu:1595-1605
        float k = (float)(sumB * 1.0 / P->pv_num);
        g->gamma = k;
        if (k > 0.1 || (k < 0.1 && (0.1 - k) < 0.01)) {
            *more = false;
            return GAHHG_OK;
        }
    }
    // capacities for the level being created
    const int vs = lv.vstart + lv.vnum, bs = lv.bstart + lv.bnum, cs = lv.cstart + lv.cnum;
    GAHHG_TRY(g->V.reserve((size_t)vs + sumA, s));
    GAHHG_TRY(g->B.reserve((size_t)bs + 7 * (size_t)sumA, s));
    GAHHG_TRY(g->C.reserve((size_t)cs + sumB + sumA, s));
    k_create_center<<<blocks_for(lv.cnum), TPB, 0, s>>>(g->V.ptr, vs, g->B.ptr, bs, g->C.ptr, lv.cstart, lv.cnum,
                                                        g->off_a.ptr, g->off_b.ptr);
    Level nl;
    nl.vstart = vs;
    nl.vnum = sumA;
    nl.bstart = bs;
    nl.bnum = sumA;
    nl.cstart = cs;
    nl.cnum = sumB;
    nl.rnum = 0;
    g->levels[L].rnum = sumB;

    GAHHG_TRY(g->cell_a.reserve(sumA, s, false));
    GAHHG_TRY(g->cell_b.reserve(sumA, s, false));
    GAHHG_TRY(g->off_a.reserve(sumA, s, false));
    GAHHG_TRY(g->off_b.reserve(sumA, s, false));
    k_border_sc_offsets<<<blocks_for(sumA), TPB, 0, s>>>(g->B.ptr, g->C.ptr, nl.bstart, sumA, g->cell_a.ptr,
                                                         g->cell_b.ptr);
    GAHHG_TRY(scan_state_reserve(&g->scan_state, sumA));
    GAHHG_TRY(scan_exclusive(g->cell_a.ptr, g->off_a.ptr, sumA, g->d_counts + HC_SUM_A2, g->scan_state, g->d_err, s));
    GAHHG_TRY(scan_exclusive(g->cell_b.ptr, g->off_b.ptr, sumA, g->d_counts + HC_SUM_B2, g->scan_state, g->d_err, s));
    k_create_border_sc<<<blocks_for(sumA), TPB, 0, s>>>(g->V.ptr, g->B.ptr, nl.bstart, sumA, g->C.ptr, nl.cstart,
                                                        sumB, g->off_a.ptr, g->off_b.ptr);
    GAHHG_CUDA_TRY(cudaGetLastError());
    GAHHG_TRY(read_counts(g));
    const int sumA2 = g->h_counts[HC_SUM_A2], sumB2 = g->h_counts[HC_SUM_B2];
    const int bsc_start = nl.cstart + nl.cnum;
    nl.cnum += sumB2;
    nl.bnum += sumA2;
    g->levels[L + 1] = nl;
    k_set_sc_partner<<<blocks_for(sumB2), TPB, 0, s>>>(g->B.ptr, g->C.ptr, bsc_start, sumB2);
    GAHHG_CUDA_TRY(cudaGetLastError());
    *more = true;
    return GAHHG_OK;
}

// GAHHG::dispatchSELast: bottom-level edge lists.
static gahhg_status dispatch_last(Grid* g)
{
    cudaStream_t s = g->stream;
    const Polygon* P = g->poly;
    const int n = P->pv_num;
    Level& last = g->levels[g->gnum - 1];
    GridView gv = view(g);
    const int level = g->gnum - 1;
    int* buf = g->edge_cur.ptr;  // cell of each edge's start vertex at level gnum-2

    k_edge_refs<WALK_COUNT><<<blocks_for(n), TPB, 0, s>>>(P->d_pv, P->d_pe, n, gv, level, g->levels[0].cnum, buf,
                                                         g->edge_cnt.ptr, nullptr, nullptr, g->d_err);
    GAHHG_TRY(scan_state_reserve(&g->scan_state, n));
    GAHHG_TRY(scan_exclusive(g->edge_cnt.ptr, g->edge_off.ptr, n, g->d_counts + HC_REFS, g->scan_state, g->d_err, s));
    GAHHG_TRY(read_counts(g));
    const int R = g->h_counts[HC_REFS];
    last.rnum = R;
    GAHHG_TRY(g->ref_cell.reserve((size_t)R + 1, s, false));
    GAHHG_TRY(g->ref_flag.reserve((size_t)R + 1, s, false));
    GAHHG_TRY(g->ref_edge.reserve((size_t)R + 1, s, false));
    GAHHG_TRY(g->refs.reserve((size_t)R + 1, s, false));
    k_edge_refs<WALK_WRITE><<<blocks_for(n), TPB, 0, s>>>(P->d_pv, P->d_pe, n, gv, level, g->levels[0].cnum, buf,
                                                         g->edge_cnt.ptr, g->edge_off.ptr, g->ref_cell.ptr, g->d_err);
    GAHHG_CUDA_TRY(cudaMemsetAsync(g->ref_flag.ptr, 0, sizeof(int) * ((size_t)R + 1), s));
    k_edge_flags<<<blocks_for(n), TPB, 0, s>>>(g->edge_off.ptr, n, g->ref_flag.ptr, R);
    GAHHG_TRY(scan_state_reserve(&g->scan_state, R));
    GAHHG_TRY(scan_exclusive(g->ref_flag.ptr, g->ref_edge.ptr, R, g->d_counts + HC_SUM_A, g->scan_state, g->d_err, s));
    k_add<<<blocks_for(R), TPB, 0, s>>>(g->ref_flag.ptr, g->ref_edge.ptr, R);

    const int cn = last.cnum;
    GAHHG_TRY(g->cell_a.reserve(cn, s, false));
    GAHHG_TRY(g->off_a.reserve(cn, s, false));
    GAHHG_TRY(g->cell_b.reserve(cn, s, false));
    GAHHG_CUDA_TRY(cudaMemsetAsync(g->cell_a.ptr, 0, sizeof(int) * cn, s));
    k_count_per_cell<<<blocks_for(R), TPB, 0, s>>>(g->ref_cell.ptr, R, last.cstart, cn, g->cell_a.ptr, g->d_err);
    GAHHG_TRY(scan_state_reserve(&g->scan_state, cn));
    GAHHG_TRY(scan_exclusive(g->cell_a.ptr, g->off_a.ptr, cn, g->d_counts + HC_SUM_B, g->scan_state, g->d_err, s));
    GAHHG_CUDA_TRY(cudaMemcpyAsync(g->cell_b.ptr, g->off_a.ptr, sizeof(int) * cn, cudaMemcpyDeviceToDevice, s));
    k_scatter_refs<<<blocks_for(R), TPB, 0, s>>>(g->ref_cell.ptr, g->ref_edge.ptr, R, last.cstart, cn, g->cell_b.ptr,
                                                 g->refs.ptr);
    k_sort_cell_refs<<<blocks_for(cn), TPB, 0, s>>>(g->C.ptr, last.cstart, cn, g->cell_a.ptr, g->off_a.ptr,
                                                    g->refs.ptr);
    GAHHG_CUDA_TRY(cudaGetLastError());
    return GAHHG_OK;
}

gahhg_status grid_alloc_common(Grid* g)
{
    if (!g->d_err) GAHHG_CUDA_TRY(cudaMalloc(&g->d_err, sizeof(DeviceErrors)));
    if (!g->d_counts) GAHHG_CUDA_TRY(cudaMalloc(&g->d_counts, 64 * sizeof(int)));
    if (!g->h_counts) GAHHG_CUDA_TRY(cudaMallocHost(&g->h_counts, 64 * sizeof(int)));
    GAHHG_CUDA_TRY(cudaMemsetAsync(g->d_err, 0, sizeof(DeviceErrors), g->stream));
    return GAHHG_OK;
}

gahhg_status grid_build(Grid* g)
{
    cudaStream_t s = g->stream;
    const Polygon* P = g->poly;
    const int n = P->pv_num;

    // createAHHGInit (source/GPISPAHHG.cu:1947-1974): level-0 grid upload
    std::vector<D3> V0;
    std::vector<Border> B0;
    std::vector<Cell> C0;
    build_grid0(V0, B0, C0);
    const int maxd = g->opts.max_depth > 0 ? g->opts.max_depth : 15;
    g->levels.assign(maxd, Level{0, 0, 0, 0, 0, 0, 0});
    g->levels[0] = Level{0, (int)V0.size(), 0, (int)B0.size(), 0, (int)C0.size(), 0};
    g->gnum = maxd;
    GAHHG_TRY(g->V.reserve(n > 160 ? n : 160, s));
    GAHHG_TRY(g->B.reserve(4 * (size_t)n > 480 ? 4 * (size_t)n : 480, s));
    GAHHG_TRY(g->C.reserve(n > 84 ? n : 84, s));
    GAHHG_TRY(g->edge_cur.reserve(n, s));
    GAHHG_TRY(g->edge_prev.reserve(n, s));
    GAHHG_TRY(g->edge_cnt.reserve(n, s));
    GAHHG_TRY(g->edge_off.reserve(n, s));
    if (!g->d_err) GAHHG_CUDA_TRY(cudaMalloc(&g->d_err, sizeof(DeviceErrors)));
    if (!g->d_counts) GAHHG_CUDA_TRY(cudaMalloc(&g->d_counts, 64 * sizeof(int)));
    if (!g->h_counts) GAHHG_CUDA_TRY(cudaMallocHost(&g->h_counts, 64 * sizeof(int)));
    GAHHG_CUDA_TRY(cudaMemsetAsync(g->d_err, 0, sizeof(DeviceErrors), s));
    GAHHG_CUDA_TRY(cudaMemsetAsync(g->edge_cur.ptr, 0, sizeof(int) * n, s));
    GAHHG_CUDA_TRY(cudaMemsetAsync(g->edge_prev.ptr, 0, sizeof(int) * n, s));
    GAHHG_CUDA_TRY(cudaMemcpyAsync(g->V.ptr, V0.data(), sizeof(D3) * V0.size(), cudaMemcpyHostToDevice, s));
    GAHHG_CUDA_TRY(cudaMemcpyAsync(g->B.ptr, B0.data(), sizeof(Border) * B0.size(), cudaMemcpyHostToDevice, s));
    GAHHG_CUDA_TRY(cudaMemcpyAsync(g->C.ptr, C0.data(), sizeof(Cell) * C0.size(), cudaMemcpyHostToDevice, s));
    GAHHG_CUDA_TRY(cudaStreamSynchronize(s));

    // createAHHG (source/GPISPAHHG.cu:1976-2015), timed like createAHHGTime
    const double t0 = now_seconds();
    bool early = false;
    for (int i = 0; i < g->gnum - 1; i++) {
        bool more = true;
        GAHHG_TRY(div_grid(g, i, &more));
        if (!more) {
            early = true;
            g->gnum = i + 1;
            break;
        }
    }
    if (g->opts.max_depth == 1) g->gamma = (float)(42 * 1.0 / n);
    if (early && g->gnum != 1) {
        // the stopping level already advanced each edge's start cell; the
        // edge lists need the cell one level up (:1999-2004)
        std::swap(g->edge_cur, g->edge_prev);
    }
    GAHHG_TRY(dispatch_last(g));
    GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
    g->stats.create_s = now_seconds() - t0;
    GAHHG_TRY(check_device_errors(g, "build"));
    g->levels.resize(g->gnum);
    return GAHHG_OK;
}

}  // namespace gahhg
