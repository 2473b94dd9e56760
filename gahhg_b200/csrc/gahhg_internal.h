// gahhg_internal.h - host-side objects behind the C ABI (include/gahhg.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "geom.cuh"
#include "gahhg.h"

namespace gahhg {

// ----------------------------------------------------------------- knobs --
// Current value of a gahhg_knob (process-wide, set by gahhg_set_knob).
long long knob(int k);

// ---------------------------------------------------------------- errors --
void set_error(const char* fmt, ...);
const char* last_error();

#define GAHHG_CUDA_TRY(expr)                                                          \
    do {                                                                              \
        cudaError_t e_ = (expr);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            ::gahhg::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr,            \
                               cudaGetErrorString(e_));                               \
            return GAHHG_ERR_CUDA;                                                    \
        }                                                                             \
    } while (0)

#define GAHHG_TRY(expr)                              \
    do {                                             \
        gahhg_status s_ = (expr);                    \
        if (s_ != GAHHG_OK) return s_;               \
    } while (0)

// Device word where kernels record problems instead of trapping: a walk that
// hit its step limit, an index that would leave its array, a scan whose
// look-back gave up.  Read by the host after each phase.
struct DeviceErrors {
    int walk_step_limit;
    int walk_bad_index;
    int scan_lookback_timeout;
    int classify_no_converge;
    int lattice_overflow;
    int other;
    int first_code;
    int first_tid;
};

// Stream-ordered scratch from a library-owned pool per device that keeps
// freed memory cached (the default pool returns it to the driver at every
// synchronisation).  Allocation and release are ordered on the given stream,
// so builds on different streams never synchronise the whole device.
gahhg_status pool_alloc(void** p, size_t bytes, int device, cudaStream_t s);
// Raises the pool's release threshold to at least `bytes` (never lowers it).
gahhg_status pool_keep(int device, size_t bytes);

// Growable device array (explicit capacity, reallocated with a copy), backed
// by the pool and ordered on the stream it was last reserved on.
template <class T> struct DevArray {
    T* ptr = nullptr;
    size_t cap = 0;
    cudaStream_t stream = nullptr;
    DevArray() = default;
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    DevArray(DevArray&& o) noexcept : ptr(o.ptr), cap(o.cap), stream(o.stream)
    {
        o.ptr = nullptr;
        o.cap = 0;
    }
    DevArray& operator=(DevArray&& o) noexcept
    {
        if (this != &o) {
            release();
            ptr = o.ptr;
            cap = o.cap;
            stream = o.stream;
            o.ptr = nullptr;
            o.cap = 0;
        }
        return *this;
    }
    // owners release explicitly before destroying the stream; this only
    // catches early returns
    ~DevArray() { release(); }
    gahhg_status reserve(size_t n, cudaStream_t s, bool keep = true)
    {
        if (n <= cap) return GAHHG_OK;
        size_t ncap = cap ? cap : 1024;
        while (ncap < n) ncap *= 2;
        int dev = 0;
        cudaGetDevice(&dev);
        T* np = nullptr;
        if (pool_alloc((void**)&np, ncap * sizeof(T), dev, s) != GAHHG_OK) {
            cudaGetLastError();
            set_error("device allocation of %zu bytes failed", ncap * sizeof(T));
            return GAHHG_ERR_NOMEM;
        }
        if (ptr) {
            if (keep) GAHHG_CUDA_TRY(cudaMemcpyAsync(np, ptr, cap * sizeof(T), cudaMemcpyDeviceToDevice, s));
            cudaFreeAsync(ptr, s);
        }
        ptr = np;
        cap = ncap;
        stream = s;
        return GAHHG_OK;
    }
    void release()
    {
        if (ptr) cudaFreeAsync(ptr, stream);
        ptr = nullptr;
        cap = 0;
    }
};

// ---------------------------------------------------------------- polygon --
struct Polygon {
    int pv_num = 0;               // number of edges == number of ring vertices
    int num_rings = 0;
    std::vector<double> lonlat;   // per vertex lon, lat (degrees, as read)
    std::vector<D3> pv;           // canonical XYZ
    std::vector<int> pe;          // edge i = (pe[2i], pe[2i+1]), oriented
    std::vector<int> ring_start;  // first vertex of each ring (num_rings + 1)
    std::string path;
    // device copies
    D3* d_pv = nullptr;
    int* d_pe = nullptr;
    bool pooled = false;          // device copies come from the stream-ordered pool
    // Device copies: synchronous cudaMalloc without a stream, else ordered on s.
    gahhg_status upload(cudaStream_t s = nullptr, int device = 0);
    void copy_host(const Polygon& o);  // host arrays only
    Polygon() = default;
    Polygon(const Polygon&) = delete;
    Polygon& operator=(const Polygon&) = delete;
    ~Polygon();
};

gahhg_status load_polygon_file(const char* path, Polygon* out);
gahhg_status polygon_from_rings(const double* lonlat, const int64_t* ring_offsets, int nrings,
                                Polygon* out);

struct Points {
    std::unique_ptr<double[]> lonlat;  // lon, lat per point (not zero-filled: every entry is parsed)
    size_t n = 0;
    std::string path;
};
gahhg_status load_points_file(const char* path, Points* out);
// Binary sidecar `<csv>.f64`: a 64-byte header (magic, point count, size
// and modification time of the CSV it was made from) and the lon/lat doubles.
gahhg_status load_points_sidecar(const char* csv_path, Points* out);  // GAHHG_ERR_STATE when absent or stale
gahhg_status write_points_sidecar(const char* csv_path, const Points& pts);

// ------------------------------------------------------------ level-0 grid --
void build_grid0(std::vector<D3>& V, std::vector<Border>& B, std::vector<Cell>& C);

// --------------------------------------------------------------- the grid --
struct Lattice;  // exact-semantics query index (lattice.cu)

struct Grid {
    const Polygon* poly = nullptr;
    gahhg_build_opts opts{};
    cudaStream_t stream = nullptr;
    cudaStream_t aux_stream = nullptr;  // second stream of the pipelined host-buffer query
    int device = 0;

    std::vector<Level> levels;    // levels[0..gnum-1]
    int gnum = 0;
    float gamma = 0.f;

    DevArray<D3> V;
    DevArray<Border> B;
    DevArray<Cell> C;
    DevArray<int> refs;           // bottom-level cell -> edge CSR
    // build scratch
    DevArray<int> cell_a, cell_b, off_a, off_b;
    DevArray<int> edge_cur, edge_prev, edge_cnt, edge_off, ref_cell, ref_flag, ref_edge;
    DevArray<int> type_old, type_cur, type_next;
    DeviceErrors* d_err = nullptr;
    int* d_counts = nullptr;      // small device header of counts
    int* h_counts = nullptr;      // pinned mirror
    void* scan_state = nullptr;   // decoupled look-back tile status

    // query-layout copies (FP64 reference-semantics query)
    void* qlayout = nullptr;
    Lattice* lattice = nullptr;

    gahhg_stats stats{};
    bool classified = false;
    bool borrowed = false;        // stream and scan state belong to a batch worker
    // the hexagon hierarchy exists (always for reference semantics; for exact
    // semantics built on first need: report, export, depth, FP64 reference query)
    bool hierarchy = false;
    std::mutex hierarchy_mu;

    ~Grid();
};

gahhg_status grid_alloc_common(Grid* g);  // device error word and count buffers
gahhg_status grid_build(Grid* g);
gahhg_status grid_classify(Grid* g);
gahhg_status grid_query_ref(Grid* g, const double* d_lonlat, size_t n, uint8_t* d_labels, cudaStream_t s,
                            uint64_t* d_counters);
gahhg_status grid_prepare_query(Grid* g);
gahhg_status check_device_errors(Grid* g, const char* phase);

// exact engine
gahhg_status lattice_build(Grid* g);
// Exact indexes of several polygons built together (shared launches); g
// lends the device, stream, scratch counts, error word and scan state.
struct GroupIndex;
gahhg_status lattice_build_group(Grid* g, Polygon* const* polys, int count, const int* top_cells,
                                 const int* leaf_edges, GroupIndex** out);
void group_free(GroupIndex* G);
void group_view_write(const GroupIndex* G, int i, void* dst);
long long group_summary_words(const GroupIndex* G, int i);
long long group_bytes(const GroupIndex* G);
gahhg_status lattice_query(Grid* g, const double* d_lonlat, size_t n, uint8_t* d_labels, int precision,
                           cudaStream_t s, uint64_t* d_counters);
gahhg_status lattice_query_noalloc(Grid* g, const double* d_lonlat, size_t n, uint8_t* d_labels, int precision,
                                   cudaStream_t s);
long long lattice_noalloc_max_points();
void lattice_free(Lattice* L);
// batches (lattice.cu)
size_t lattice_view_bytes();
size_t batch_chunk_bytes();
void lattice_view_write(const Grid* g, void* dst);
long long lattice_summary_words(const Grid* g);
// Locate blocks on `device` whose summary copy ran out of time (plain loads instead).
gahhg_status lattice_staging_fallbacks(int device, unsigned long long* out);
// Chunks over segments of points stored segment after segment; segment p's
// points belong to view seg_view[p] (p itself when seg_view is null).
void batch_make_chunks(const long long* offsets, int nseg, int chunk_points, const int* swords, const int* seg_view,
                       std::vector<uint8_t>& out, int* nchunks);
void batch_write_chunks(const long long* offsets, int nseg, int chunk_points, const int* swords, const int* seg_view,
                        void* out, int* nchunks);
size_t batch_chunk_count_bound(long long points, int nseg, int chunk_points);
// Words of a batch queue whose pass-2 part holds queue_cap points (with their
// leaf words; the escalation queues and theirs follow).
size_t batch_queue_words(long long queue_cap);
// counters[0..4] must be zero on entry unless zero_counters is set.  shape
// indexes the pass-1 launch shapes (batch_shape_info).
gahhg_status batch_query_launch(const void* d_views, const void* d_chunks, int nchunks, const double* d_lonlat,
                                uint8_t* d_labels, int precision, uint32_t* queue, long long queue_cap,
                                unsigned int* counters, uint64_t* d_stats, cudaStream_t s, int device,
                                bool zero_counters = true, int shape = 0);
int batch_shape_count();
bool batch_shape_info(int shape, int* points_per_thread, int* blocks_per_sm);
size_t lattice_bytes(const Lattice* L);
size_t lattice_device_bytes(const Lattice* L);  // capacity held on the device

// scans (scan.cu)
size_t scan_state_bytes(size_t n);
gahhg_status scan_state_reserve(void** state, size_t max_n);
void scan_state_destroy(void* state);
gahhg_status scan_exclusive(const int* d_in, int* d_out, int n, int* d_total, void* state, DeviceErrors* err,
                            cudaStream_t s);

double now_seconds();

// Host threads with one non-blocking stream and look-back scan state each,
// building exact indexes concurrently (batch.cpp).
struct WorkerPool {
    int device = 0;
    std::vector<cudaStream_t> streams;
    std::vector<void*> scans;
    gahhg_status create(int device, int n, int priority = 0);
    void destroy();
    gahhg_status build_all(const std::vector<Polygon*>& polys, const gahhg_build_opts& base, const int* top,
                           const int* leaf, std::vector<Grid*>& grids, int* failed);
};
gahhg_status build_exact_grid(Polygon* P, int device, cudaStream_t s, void** scan, const gahhg_build_opts& base,
                              int top, int leaf, Grid** out);

}  // namespace gahhg

struct gahhg_polygon { gahhg::Polygon p; };
struct gahhg_points { gahhg::Points p; };
struct gahhg_grid { gahhg::Grid g; };
