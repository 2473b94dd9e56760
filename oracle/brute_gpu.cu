/*
 * brute_gpu.cu - the exact oracle's brute force over every edge, on the GPU
 * (TEST INFRASTRUCTURE: only tests/ load it).
 *
 * Computes the labels that oracle/exact_pip.c defines (label_xyz), for
 * point sets far too large for the CPU: a point takes the label of its
 * nearest hub XOR the parity of the polygon edges crossing arc(hub, q), with
 * a point equal to a polygon vertex inside.  The crossing test is the
 * oracle's (oracle_crossing with r = hub):
 *     acb = -orient(a, b, H), bda = orient(a, b, q),
 *     cbd = -orient(H, q, b), dac = orient(H, q, a),  crossing iff all equal.
 * orient(a, b, H) is the CPU oracle's exact sign (computed there, passed in);
 * the other three are evaluated here in FP64 with a forward error bound, and
 * a point any of whose signs falls within its bound (or that meets a hub
 * coinciding with a vertex) is reported undecided (label 0), for the CPU
 * oracle to label.  Every decided sign is the exact sign, so every decided
 * label equals the CPU oracle's.
 *
 * The predicates are written here from the determinant identities below and
 * share no code with the library's kernels (only the canonical lon/lat
 * conversion of include/gahhg_canon.h, which defines the points):
 *   det[a; b; q] = det[a; u; v] = v . (a x u),  u = b - a, v = q - a
 *   det[H; q; x] = z . (H x q),                  z = x - q
 * (row operations; the small translated rows keep the error relative to the
 * edge's length and the point's distance, not to the unit sphere).
 *
 * Error bound (eps = 2^-53, every operation separately rounded: built with
 * --fmad=false).  With u, v the rounded differences, N = fl(a x u) and
 * P_i = |a_j u_k| + |a_k u_j| ((i, j, k) cyclic):
 *   |fl(N . v) - det[a; b; q]|
 *     <= (3.01 [dot] + 2.01 [N] + 1.01 [rounding of v] + 1.03 [of u]) eps
 *        * sum_i P_i |v_i|   <  10 eps sum_i P_i |v_i|
 * and the same for z . (H x q) with PW_i = |H_j q_k| + |H_k q_j| (no u term:
 * 6.03 eps; 10 eps used as well).  The bound's own rounding (a few eps
 * relative) is inside the margin.  A sign is taken only when |value| > bound;
 * an exact zero is never decided here (the CPU oracle breaks it by
 * simulation of simplicity).
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "gahhg_canon.h"

namespace {

constexpr double EPS = 1.1102230246251565e-16;  // 2^-53
constexpr double BOUND = 10.0 * EPS;
constexpr int TPB = 128;
constexpr int PPT = 2;       // points per thread (edge loads shared)
constexpr int TILE = 256;    // edges per shared-memory tile

// One edge, laid out for 16-byte shared-memory loads.
struct __align__(16) EdgeRec {
    double2 r0;  // a0, a1
    double2 r1;  // a2, N0
    double2 r2;  // N1, N2
    double2 r3;  // P0, P1
    double2 r4;  // P2, b0
    double2 r5;  // b1, b2
    int flags;   // bit 0: zero-length edge (no crossing test); bits 8..13: hub k is an end of the edge
    int side;    // 2 bits per hub k: orient(a, b, H_k) as 1 -> +1, 2 -> -1, 0 -> 0
    int pad[2];
};
static_assert(sizeof(EdgeRec) == 112, "EdgeRec");

struct Hubs {
    double h[6][3];
    int label[6];
};

struct PointState {
    double q[3];
    double W[3], PW[3];  // H x q and its bound terms
    int hub;
    int par;
    bool amb, vert;
};

__host__ __device__ __forceinline__ void point_init(PointState& S, const Hubs& H, double lon, double lat)
{
    S.amb = false;
    S.vert = false;
    S.par = 0;
    S.hub = 0;
    gahhg_canon_query_xyz(lon, lat, S.q);
    // nearest hub: the first maximum of the dot product, as the CPU oracle
    double bd = -1e300;
    for (int k = 0; k < 6; k++) {
        const double d = H.h[k][0] * S.q[0] + H.h[k][1] * S.q[1] + H.h[k][2] * S.q[2];
        if (d > bd) {
            bd = d;
            S.hub = k;
        }
    }
    const double* h = H.h[S.hub];
    S.W[0] = h[1] * S.q[2] - h[2] * S.q[1];
    S.W[1] = h[2] * S.q[0] - h[0] * S.q[2];
    S.W[2] = h[0] * S.q[1] - h[1] * S.q[0];
    S.PW[0] = fabs(h[1] * S.q[2]) + fabs(h[2] * S.q[1]);
    S.PW[1] = fabs(h[2] * S.q[0]) + fabs(h[0] * S.q[2]);
    S.PW[2] = fabs(h[0] * S.q[1]) + fabs(h[1] * S.q[0]);
}

__host__ __device__ __forceinline__ int hub_side(int side, int k)
{
    const int c = (side >> (2 * k)) & 3;
    return c == 1 ? 1 : (c == 2 ? -1 : 0);
}

// One edge's contribution to a point: vertex rule, crossing parity, or
// "undecided" when a sign is within its bound.
__host__ __device__ __forceinline__ void point_edge(PointState& S, const EdgeRec& e)
{
    const double2 r0 = e.r0, r1 = e.r1;
    const double a0 = r0.x, a1 = r0.y, a2 = r1.x;
    if (S.q[0] == a0 && S.q[1] == a1 && S.q[2] == a2) S.vert = true;  // vertex rule
    const int flags = e.flags;
    if (flags & 1) return;               // zero-length edge
    if (flags & (256 << S.hub)) {        // the hub is an end of the edge
        S.amb = true;
        return;
    }
    // bda = orient(a, b, q) = v . (a x u)
    const double2 r2 = e.r2, r3 = e.r3, r4 = e.r4;
    const double v0 = S.q[0] - a0, v1 = S.q[1] - a1, v2 = S.q[2] - a2;
    const double d = v0 * r1.y + v1 * r2.x + v2 * r2.y;
    const double bd = BOUND * (r3.x * fabs(v0) + r3.y * fabs(v1) + r4.x * fabs(v2));
    if (!(fabs(d) > bd)) {
        S.amb = true;
        return;
    }
    const int bda = d > 0.0 ? 1 : -1;
    const int acb = -hub_side(e.side, S.hub);
    if (acb == 0) {
        S.amb = true;
        return;
    }
    if (bda != acb) return;
    // cbd = -orient(H, q, b) = -(b - q) . (H x q)
    const double2 r5 = e.r5;
    const double z0 = r4.y - S.q[0], z1 = r5.x - S.q[1], z2 = r5.y - S.q[2];
    const double db = z0 * S.W[0] + z1 * S.W[1] + z2 * S.W[2];
    const double bb = BOUND * (S.PW[0] * fabs(z0) + S.PW[1] * fabs(z1) + S.PW[2] * fabs(z2));
    if (!(fabs(db) > bb)) {
        S.amb = true;
        return;
    }
    if ((db > 0.0 ? -1 : 1) != acb) return;
    // dac = orient(H, q, a) = (a - q) . (H x q)
    const double y0 = a0 - S.q[0], y1 = a1 - S.q[1], y2 = a2 - S.q[2];
    const double da = y0 * S.W[0] + y1 * S.W[1] + y2 * S.W[2];
    const double ba = BOUND * (S.PW[0] * fabs(y0) + S.PW[1] * fabs(y1) + S.PW[2] * fabs(y2));
    if (!(fabs(da) > ba)) {
        S.amb = true;
        return;
    }
    if ((da > 0.0 ? 1 : -1) == acb) S.par ^= 1;
}

__host__ __device__ __forceinline__ uint8_t point_label(const PointState& S, const Hubs& H)
{
    const double* h = H.h[S.hub];
    if (S.vert) return 2;
    if (S.q[0] == h[0] && S.q[1] == h[1] && S.q[2] == h[2]) return (uint8_t)H.label[S.hub];
    if (S.amb) return 0;
    return (uint8_t)(S.par ? 3 - H.label[S.hub] : H.label[S.hub]);
}

__global__ void __launch_bounds__(TPB) k_brute(const EdgeRec* __restrict__ E, int n, Hubs H,
                                               const double2* __restrict__ ll, long long np,
                                               uint8_t* __restrict__ out)
{
    __shared__ EdgeRec s[TILE];
    PointState P[PPT];
    const long long base = ((long long)blockIdx.x * TPB + threadIdx.x) * PPT;
#pragma unroll
    for (int j = 0; j < PPT; j++) {
        const double2 p = base + j < np ? ll[base + j] : make_double2(0.0, 0.0);
        point_init(P[j], H, p.x, p.y);
    }
    for (int t0 = 0; t0 < n; t0 += TILE) {
        const int m = min(TILE, n - t0);
        __syncthreads();
        for (int k = threadIdx.x; k < m; k += TPB) s[k] = E[t0 + k];
        __syncthreads();
        for (int k = 0; k < m; k++) {
#pragma unroll
            for (int j = 0; j < PPT; j++) point_edge(P[j], s[k]);
        }
    }
#pragma unroll
    for (int j = 0; j < PPT; j++)
        if (base + j < np) out[base + j] = point_label(P[j], H);
}

#define BRUTE_TRY(x)                                                                   \
    do {                                                                               \
        cudaError_t e_ = (x);                                                          \
        if (e_ != cudaSuccess) {                                                       \
            fprintf(stderr, "brute_gpu: %s: %s\n", #x, cudaGetErrorString(e_));        \
            rc = -1;                                                                   \
            goto done;                                                                 \
        }                                                                              \
    } while (0)

}  // namespace

/*
 * Labels of `np` points (lon, lat pairs) against the polygon with vertices
 * pv (canonical XYZ) and edges pe (2 per edge, n edges).  side[6 e + k] =
 * orient(a_e, b_e, hub_k) from the CPU oracle; hubs and hub_label from its
 * exact_poly_info.  labels get 1 (out), 2 (in) or 0 (undecided here).
 * Returns the number of undecided points, or -1 on a CUDA error.
 */
static void make_records(const double* pv, const int* pe, int n, const signed char* side, const double* hubs,
                         const int* hub_label, std::vector<EdgeRec>& E, Hubs& H)
{
    E.resize((size_t)n);
    for (int k = 0; k < 6; k++) {
        for (int c = 0; c < 3; c++) H.h[k][c] = hubs[3 * k + c];
        H.label[k] = hub_label[k];
    }
    for (int e = 0; e < n; e++) {
        const double* a = pv + 3 * (size_t)pe[2 * e];
        const double* b = pv + 3 * (size_t)pe[2 * e + 1];
        const double u0 = b[0] - a[0], u1 = b[1] - a[1], u2 = b[2] - a[2];
        EdgeRec& r = E[e];
        memset(&r, 0, sizeof(r));
        r.r0 = make_double2(a[0], a[1]);
        r.r1 = make_double2(a[2], a[1] * u2 - a[2] * u1);
        r.r2 = make_double2(a[2] * u0 - a[0] * u2, a[0] * u1 - a[1] * u0);
        r.r3 = make_double2(fabs(a[1] * u2) + fabs(a[2] * u1), fabs(a[2] * u0) + fabs(a[0] * u2));
        r.r4 = make_double2(fabs(a[0] * u1) + fabs(a[1] * u0), b[0]);
        r.r5 = make_double2(b[1], b[2]);
        const bool zero = a[0] == b[0] && a[1] == b[1] && a[2] == b[2];
        r.flags = zero ? 1 : 0;
        for (int k = 0; k < 6; k++) {
            const double* h = hubs + 3 * k;
            const bool on = (h[0] == a[0] && h[1] == a[1] && h[2] == a[2]) ||
                            (h[0] == b[0] && h[1] == b[1] && h[2] == b[2]);
            if (on) r.flags |= 256 << k;
            const int sd = side[6 * (size_t)e + k];
            r.side |= (sd > 0 ? 1 : (sd < 0 ? 2 : 0)) << (2 * k);
        }
    }
}

/*
 * Labels of `np` points (lon, lat pairs) against the polygon with vertices
 * pv (canonical XYZ) and edges pe (2 per edge, n edges).  side[6 e + k] =
 * orient(a_e, b_e, hub_k) from the CPU oracle; hubs and hub_label from its
 * exact_poly_info.  labels get 1 (out), 2 (in) or 0 (undecided here).
 * Returns the number of undecided points, or -1 on a CUDA error.
 */
extern "C" long long brute_gpu_label(const double* pv, const int* pe, int n, const signed char* side,
                                     const double* hubs, const int* hub_label, const double* lonlat,
                                     long long np, uint8_t* labels, int device)
{
    long long rc = 0;
    EdgeRec* dE = nullptr;
    double2* dll = nullptr;
    uint8_t* dout = nullptr;
    const long long CH = 1LL << 24;
    std::vector<EdgeRec> E;
    Hubs H;
    make_records(pv, pe, n, side, hubs, hub_label, E, H);
    const long long chunk = np < CH ? np : CH;
    BRUTE_TRY(cudaSetDevice(device));
    if (n > 0) BRUTE_TRY(cudaMalloc(&dE, sizeof(EdgeRec) * (size_t)n));
    if (chunk > 0) {
        BRUTE_TRY(cudaMalloc(&dll, sizeof(double2) * (size_t)chunk));
        BRUTE_TRY(cudaMalloc(&dout, (size_t)chunk));
    }
    if (n > 0) BRUTE_TRY(cudaMemcpy(dE, E.data(), sizeof(EdgeRec) * (size_t)n, cudaMemcpyHostToDevice));
    for (long long off = 0; off < np; off += chunk) {
        const long long m = np - off < chunk ? np - off : chunk;
        BRUTE_TRY(cudaMemcpy(dll, lonlat + 2 * off, sizeof(double2) * (size_t)m, cudaMemcpyHostToDevice));
        const long long per_block = (long long)TPB * PPT;
        const unsigned grid = (unsigned)((m + per_block - 1) / per_block);
        k_brute<<<grid, TPB>>>(dE, n, H, dll, m, dout);
        BRUTE_TRY(cudaGetLastError());
        BRUTE_TRY(cudaMemcpy(labels + off, dout, (size_t)m, cudaMemcpyDeviceToHost));
    }
    for (long long i = 0; i < np; i++) rc += labels[i] == 0;
done:
    cudaFree(dE);
    cudaFree(dll);
    cudaFree(dout);
    return rc;
}

/* The same per-point steps on the host (one thread), so that the CPU tests
 * can check them against the CPU oracle without a GPU.  Same return value. */
extern "C" long long brute_host_label(const double* pv, const int* pe, int n, const signed char* side,
                                      const double* hubs, const int* hub_label, const double* lonlat,
                                      long long np, uint8_t* labels)
{
    std::vector<EdgeRec> E;
    Hubs H;
    make_records(pv, pe, n, side, hubs, hub_label, E, H);
    long long rc = 0;
    for (long long i = 0; i < np; i++) {
        PointState S;
        point_init(S, H, lonlat[2 * i], lonlat[2 * i + 1]);
        for (int e = 0; e < n; e++) point_edge(S, E[e]);
        labels[i] = point_label(S, H);
        rc += labels[i] == 0;
    }
    return rc;
}
