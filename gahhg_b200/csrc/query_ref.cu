// query_ref.cu - point queries with the reference's semantics (FP64).
//
// kernel_PISP (source/GPISPAHHG.cu:1422-1504): locate the point among the 42
// level-0 cells, descend through center and border subcells, and in a leaf
// with edges count crossings of arc(cell center, p) with each edge
// (device_isEEInter :351-378, epsilon rules included).
//
// Same arithmetic, different memory layout: borders are repacked into 32-byte
// records (normal + subcell, one sector per plane test), cells into 32-byte
// records, and the per-edge great-circle normal and per-leaf center are
// computed once at preparation with the exact operations the reference
// repeats per point, so labels are unchanged bit for bit.  Input is lon/lat
// (16 B/point), converted on the device with the canonical conversion
// (FakeLL2XYZ semantics, gahhg_canon.h); output is one byte per point.
#include "gahhg_canon.h"
#include "gahhg_internal.h"

namespace gahhg {

namespace {

struct __align__(32) QBorder {
    double n[3];
    int subcell;
    int pad;
};
struct __align__(32) QCell {
    int bstart, bnum, subcell, rnum;
    int rstart, type, pad0, pad1;
};
struct QEdge {
    D3 p0, p1, n;
};

struct QueryView {
    const QBorder* B;
    const QCell* C;
    const D3* center;
    const QEdge* E;
    const int* refs;
};

struct QLayout {
    DevArray<QBorder> B;
    DevArray<QCell> C;
    DevArray<D3> center;
    DevArray<QEdge> E;
};

constexpr int TPB = 256;

__global__ void k_prep_borders(const Border* B, int nb, QBorder* out)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb) return;
    QBorder q;
    q.n[0] = B[t].n[0];
    q.n[1] = B[t].n[1];
    q.n[2] = B[t].n[2];
    q.subcell = B[t].subcell;
    q.pad = 0;
    out[t] = q;
}

__global__ void k_prep_cells(const Cell* C, const Border* B, const D3* V, int nc, QCell* out, D3* center)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nc) return;
    const Cell c = C[t];
    QCell q;
    q.bstart = c.bstart;
    q.bnum = c.bnum;
    q.subcell = c.subcell;
    q.rnum = c.rnum;
    q.rstart = c.rstart;
    q.type = c.type;
    q.pad0 = q.pad1 = 0;
    out[t] = q;
    // center as kernel_PISP computes it (source/GPISPAHHG.cu:1481-1485)
    D3 s = d3(0.0, 0.0, 0.0);
    for (int i = 0; i < c.bnum; i++) s = s + V[B[c.bstart + i].v[0]];
    s = s / (double)c.bnum;
    center[t] = normalize(s);
}

__global__ void k_prep_edges(const D3* pv, const int* pe, int n, QEdge* out)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    QEdge e;
    e.p0 = pv[pe[2 * t]];
    e.p1 = pv[pe[2 * t + 1]];
    e.n = normalize(cross(e.p0, e.p1 - e.p0));
    out[t] = e;
}

__device__ __forceinline__ bool q_inside(D3 p, int cid, const QueryView& q)
{
    const QCell c = q.C[cid];
    for (int i = 0; i < c.bnum; i++) {
        const QBorder b = q.B[c.bstart + i];
        double ret = b.n[0] * p.x + b.n[1] * p.y + b.n[2] * p.z;
        if (ret < -POSITION_EPSILON) return false;
    }
    return true;
}

__device__ __forceinline__ uint8_t classify_point(D3 p, const QueryView& q)
{
    int cur = -1;
    for (int i = 0; i < 42; i++)
        if (q_inside(p, i, q)) {
            cur = i;
            break;
        }
    if (cur == -1) return 0;
    for (int depth = 0; depth < 64; depth++) {
        const QCell c = q.C[cur];
        if (c.subcell == -1) break;
        if (q_inside(p, c.subcell, q)) {
            cur = c.subcell;
            continue;
        }
        bool found = false;
        for (int i = 0; i < c.bnum; i++) {
            const int tc = q.B[c.bstart + i].subcell;
            if (tc == -1) continue;
            if (q_inside(p, tc, q)) {
                cur = tc;
                found = true;
                break;
            }
        }
        if (!found) return 0;
    }
    const QCell c = q.C[cur];
    if (c.rnum == 0) return (uint8_t)c.type;
    const D3 center = q.center[cur];
    const D3 np = normalize(cross(center, p - center));
    int count = 0;
    for (int i = 0; i < c.rnum; i++) {
        const QEdge e = q.E[q.refs[c.rstart + i]];
        double r0 = dot(np, e.p0), r1 = dot(np, e.p1);
        double r2 = dot(e.n, center), r3 = dot(e.n, p);
        bool miss = (less_zero(r0) && less_zero(r1)) || (gre_zero(r0) && gre_zero(r1)) ||
                    (less_zero(r2) && less_zero(r3)) || (gre_zero(r2) && gre_zero(r3));
        if (!miss) count++;
    }
    return (uint8_t)((count & 1) == 0 ? c.type : 3 - c.type);
}

__global__ void __launch_bounds__(TPB) k_query_ref(const double2* __restrict__ lonlat, long long n,
                                                   uint8_t* __restrict__ out, QueryView q,
                                                   unsigned long long* inside_count)
{
    const long long stride = (long long)gridDim.x * blockDim.x;
    int inside = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double2 ll = lonlat[i];
        double xyz[3];
        gahhg_canon_query_xyz(ll.x, ll.y, xyz);
        const uint8_t lab = classify_point(d3(xyz[0], xyz[1], xyz[2]), q);
        out[i] = lab;
        inside += lab == CELL_IN;
    }
    if (inside_count) {
        __shared__ int s_sum;
        if (threadIdx.x == 0) s_sum = 0;
        __syncthreads();
        for (int d = 16; d > 0; d >>= 1) inside += __shfl_down_sync(0xffffffffu, inside, d);
        if ((threadIdx.x & 31) == 0 && inside) atomicAdd(&s_sum, inside);
        __syncthreads();
        if (threadIdx.x == 0 && s_sum) atomicAdd(inside_count, (unsigned long long)s_sum);
    }
}

}  // namespace

gahhg_status grid_prepare_query(Grid* g)
{
    if (g->qlayout) return GAHHG_OK;
    cudaStream_t s = g->stream;
    QLayout* L = new QLayout();
    const Level& last = g->levels[g->gnum - 1];
    const int nb = last.bstart + last.bnum, nc = last.cstart + last.cnum, ne = g->poly->pv_num;
    gahhg_status st;
    if ((st = L->B.reserve(nb, s, false)) != GAHHG_OK || (st = L->C.reserve(nc, s, false)) != GAHHG_OK ||
        (st = L->center.reserve(nc, s, false)) != GAHHG_OK || (st = L->E.reserve(ne, s, false)) != GAHHG_OK) {
        delete L;
        return st;
    }
    k_prep_borders<<<(nb + TPB - 1) / TPB, TPB, 0, s>>>(g->B.ptr, nb, L->B.ptr);
    k_prep_cells<<<(nc + TPB - 1) / TPB, TPB, 0, s>>>(g->C.ptr, g->B.ptr, g->V.ptr, nc, L->C.ptr, L->center.ptr);
    k_prep_edges<<<(ne + TPB - 1) / TPB, TPB, 0, s>>>(g->poly->d_pv, g->poly->d_pe, ne, L->E.ptr);
    GAHHG_CUDA_TRY(cudaGetLastError());
    GAHHG_CUDA_TRY(cudaStreamSynchronize(s));
    g->qlayout = L;
    return GAHHG_OK;
}

void free_query_layout(void* p)
{
    QLayout* L = (QLayout*)p;
    if (!L) return;
    L->B.release();
    L->C.release();
    L->center.release();
    L->E.release();
    delete L;
}

size_t query_layout_bytes(const void* p)
{
    const QLayout* L = (const QLayout*)p;
    if (!L) return 0;
    return L->B.cap * sizeof(QBorder) + L->C.cap * sizeof(QCell) + L->center.cap * sizeof(D3) +
           L->E.cap * sizeof(QEdge);
}

gahhg_status grid_query_ref(Grid* g, const double* d_lonlat, size_t n, uint8_t* d_labels, cudaStream_t s,
                            uint64_t* d_counters)
{
    GAHHG_TRY(grid_prepare_query(g));
    if (n == 0) return GAHHG_OK;
    QLayout* L = (QLayout*)g->qlayout;
    QueryView q{L->B.ptr, L->C.ptr, L->center.ptr, L->E.ptr, g->refs.ptr};
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
    long long want = ((long long)n + TPB - 1) / TPB;
    int grid = (int)(want < (long long)sms * 16 ? want : (long long)sms * 16);
    k_query_ref<<<grid, TPB, 0, s>>>((const double2*)d_lonlat, (long long)n, d_labels, q,
                                     d_counters ? (unsigned long long*)d_counters + 3 : nullptr);
    GAHHG_CUDA_TRY(cudaGetLastError());
    return GAHHG_OK;
}

}  // namespace gahhg
