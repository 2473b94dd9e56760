// scan.cu - single-pass exclusive prefix sum with decoupled look-back
// (Merrill & Garland, "Single-pass Parallel Prefix Scan with Decoupled
// Look-back", NVIDIA technical report NVR-2016-002).
//
// Replaces the reference's vendored multi-pass Blelloch scan
// (source/scan/scan.cu:104-171), which allocates and frees block-sum arrays on
// every call.  One launch per scan; no allocation per call; the grand total is
// written to device memory so the host can read it in the same round trip as
// other counts.
//
// Tile status words are 64 bits: [63:34] epoch of the call, [33:32] state
// (1 = tile aggregate, 2 = inclusive prefix), [31:0] value.  A word from an
// older call has a different epoch and reads as "not ready", so the status
// array never needs clearing.  Tiles take their index from an atomic counter
// in launch order, so every tile a look-back waits on has already started;
// each wait is still bounded (spin_limit polls): when it runs out, the tile
// sums the late tile's inputs itself and goes on looking back, so the result
// stays exact, and the event is counted in DeviceErrors (scan fallbacks).
#include "gahhg_internal.h"

namespace gahhg {

namespace {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

struct ScanState {
    unsigned long long* status;
    unsigned int* counter;
    size_t max_tiles;
    unsigned int tile_base;
    unsigned int epoch;
};

__device__ __forceinline__ unsigned long long load_status(const unsigned long long* p)
{
    return *(const volatile unsigned long long*)p;
}

__global__ void __launch_bounds__(SCAN_THREADS)
k_scan_exclusive(const int* __restrict__ in, int* __restrict__ out, int n, int* total,
                 unsigned long long* status, unsigned int* counter, unsigned int tile_base,
                 unsigned int epoch, int ntiles, DeviceErrors* err, long long spin_limit)
{
    __shared__ int s_tile;
    __shared__ int s_prefix;
    __shared__ int s_warp[SCAN_THREADS / 32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) s_tile = (int)(atomicAdd(counter, 1u) - tile_base);
    __syncthreads();
    const int tile = s_tile;
    const long long base = (long long)tile * SCAN_TILE + (long long)t * SCAN_ITEMS;

    int v[SCAN_ITEMS];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        long long idx = base + k;
        v[k] = idx < n ? in[idx] : 0;
        sum += v[k];
    }
    // block-wide exclusive scan of the per-thread sums
    int incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        int w = lane < SCAN_THREADS / 32 ? s_warp[lane] : 0;
        int wi = w;
#pragma unroll
        for (int d = 1; d < SCAN_THREADS / 32; d <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, wi, d);
            if (lane >= d) wi += y;
        }
        if (lane < SCAN_THREADS / 32) s_warp[lane] = wi - w;  // exclusive warp offsets
    }
    __syncthreads();
    const int thread_excl = s_warp[warp] + incl - sum;

    if (t == SCAN_THREADS - 1) {
        const int agg = thread_excl + sum;  // block total
        const unsigned long long tagA = ((unsigned long long)((epoch << 2) | 1u)) << 32;
        const unsigned long long tagP = ((unsigned long long)((epoch << 2) | 2u)) << 32;
        int excl = 0;
        if (tile == 0) {
            atomicExch(&status[tile], tagP | (unsigned int)agg);
        } else {
            atomicExch(&status[tile], tagA | (unsigned int)agg);
            int j = tile - 1;
            long long spins = 0;
            while (j >= 0) {
                unsigned long long w = load_status(&status[j]);
                unsigned int hi = (unsigned int)(w >> 32);
                unsigned int state = hi & 3u;
                if ((hi >> 2) != (epoch & 0x3fffffffu) || state == 0u) {
                    if (++spins > spin_limit) {
                        // tile j is late: add its inputs directly and look further back
                        atomicAdd(&err->scan_lookback_timeout, 1);
                        const long long j0 = (long long)j * SCAN_TILE;
                        const long long j1 = j0 + SCAN_TILE < n ? j0 + SCAN_TILE : n;
                        int agg_j = 0;
                        for (long long idx = j0; idx < j1; idx++) agg_j += in[idx];
                        excl += agg_j;
                        spins = 0;
                        j--;
                        continue;
                    }
                    if (spins > 64) __nanosleep(64);
                    continue;
                }
                excl += (int)(unsigned int)w;
                if (state == 2u) break;
                j--;
            }
            atomicExch(&status[tile], tagP | (unsigned int)(excl + agg));
        }
        s_prefix = excl;
        if (tile == ntiles - 1) *total = excl + agg;
    }
    __syncthreads();
    int running = s_prefix + thread_excl;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        long long idx = base + k;
        if (idx < n) out[idx] = running;
        running += v[k];
    }
}

}  // namespace

size_t scan_state_bytes(size_t n)
{
    size_t tiles = (n + SCAN_TILE - 1) / SCAN_TILE + 1;
    return sizeof(ScanState) + 256 + tiles * sizeof(unsigned long long);
}

// `state` points to a host-side ScanState allocated by scan_state_create.
gahhg_status scan_state_create(void** state, size_t max_n)
{
    ScanState* st = new ScanState();
    st->max_tiles = (max_n + SCAN_TILE - 1) / SCAN_TILE + 1;
    if (cudaMalloc(&st->status, st->max_tiles * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&st->counter, sizeof(unsigned int)) != cudaSuccess) {
        set_error("scan state allocation failed");
        delete st;
        return GAHHG_ERR_NOMEM;
    }
    cudaMemset(st->status, 0, st->max_tiles * sizeof(unsigned long long));
    cudaMemset(st->counter, 0, sizeof(unsigned int));
    st->tile_base = 0;
    st->epoch = 1;
    *state = st;
    return GAHHG_OK;
}

void scan_state_destroy(void* state)
{
    ScanState* st = (ScanState*)state;
    if (!st) return;
    cudaFree(st->status);
    cudaFree(st->counter);
    delete st;
}

gahhg_status scan_state_reserve(void** state, size_t max_n)
{
    ScanState* st = (ScanState*)*state;
    size_t need = (max_n + SCAN_TILE - 1) / SCAN_TILE + 1;
    if (st && st->max_tiles >= need) return GAHHG_OK;
    // growing: the new array starts cleared and the epoch sequence continues
    unsigned int epoch = st ? st->epoch : 1, base = st ? st->tile_base : 0;
    unsigned int* counter = st ? st->counter : nullptr;
    if (st) {
        cudaFree(st->status);
        st->status = nullptr;
    } else {
        st = new ScanState();
        if (cudaMalloc(&counter, sizeof(unsigned int)) != cudaSuccess) {
            delete st;
            set_error("scan state allocation failed");
            return GAHHG_ERR_NOMEM;
        }
        cudaMemset(counter, 0, sizeof(unsigned int));
    }
    st->max_tiles = need * 2;
    if (cudaMalloc(&st->status, st->max_tiles * sizeof(unsigned long long)) != cudaSuccess) {
        set_error("scan state allocation failed");
        return GAHHG_ERR_NOMEM;
    }
    cudaMemset(st->status, 0, st->max_tiles * sizeof(unsigned long long));
    st->counter = counter;
    st->epoch = epoch;
    st->tile_base = base;
    *state = st;
    return GAHHG_OK;
}

gahhg_status scan_exclusive(const int* d_in, int* d_out, int n, int* d_total, void* state, DeviceErrors* err,
                            cudaStream_t s)
{
    if (n <= 0) {
        GAHHG_CUDA_TRY(cudaMemsetAsync(d_total, 0, sizeof(int), s));
        return GAHHG_OK;
    }
    ScanState* st = (ScanState*)state;
    const int ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if ((size_t)ntiles > st->max_tiles) {
        set_error("scan of %d items exceeds the reserved tile status (%zu tiles)", n, st->max_tiles);
        return GAHHG_ERR_CAPACITY;
    }
    const unsigned int epoch = st->epoch & 0x3fffffffu;
    k_scan_exclusive<<<ntiles, SCAN_THREADS, 0, s>>>(d_in, d_out, n, d_total, st->status, st->counter,
                                                     st->tile_base, epoch, ntiles, err,
                                                     knob(GAHHG_KNOB_SCAN_SPIN_LIMIT));
    GAHHG_CUDA_TRY(cudaGetLastError());
    st->tile_base += (unsigned int)ntiles;
    st->epoch = (st->epoch + 1) & 0x3fffffffu;
    if (st->epoch == 0) st->epoch = 1;
    return GAHHG_OK;
}

}  // namespace gahhg
