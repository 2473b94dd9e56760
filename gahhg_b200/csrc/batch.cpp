// batch.cpp - many polygons: concurrent builds, one persistent query launch,
// CUDA-graph replay.
//
// No counterpart in the reference (one polygon per process,
// source/GPISP.cu:15-70).  Builds run in groups of consecutive polygons
// (lattice_build_group: every step once for all polygons of a group, so
// launches and host round trips scale with levels, not polygons) on a pool of
// host threads, each with its own non-blocking stream and look-back scan
// state; device memory comes from the stream-ordered pool, so no build
// synchronises the device.
// A query takes all polygons' points at once (polygon after polygon) and
// runs pass 1 as one persistent launch over chunks of points.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <thread>

#include "gahhg_internal.h"

using namespace gahhg;

struct gahhg_batch {
    int device = 0;
    int count = 0;
    int chunk_points = 4096;
    int shape = 0;  // pass-1 launch shape (batch_shape_info)
    std::vector<Polygon*> polys;
    std::vector<Grid*> grids;
    std::vector<GroupIndex*> groups;  // polygons built together, in order
    std::vector<int> swords;  // summary words per polygon (chunk sizing)
    DevArray<uint8_t> views;
    WorkerPool pool;
    gahhg_batch_stats stats{};
    // graph replay state
    cudaGraphExec_t exec = nullptr;
    cudaStream_t graph_stream = nullptr;
    const double* g_lonlat = nullptr;
    uint8_t* g_labels = nullptr;
    int g_precision = -1;
    std::vector<int64_t> g_offsets;
    DevArray<uint8_t> g_chunks;
    DevArray<uint32_t> g_queue;
    DevArray<unsigned int> g_counters;
    int g_nchunks = 0;
    long long g_qcap = 0;
    cudaStream_t owner_stream = nullptr;  // stream for workspace allocations

    ~gahhg_batch()
    {
        cudaSetDevice(device);
        if (exec) cudaGraphExecDestroy(exec);
        g_chunks.release();
        g_queue.release();
        g_counters.release();
        views.release();
        for (Grid* g : grids) delete g;
        for (GroupIndex* G : groups) group_free(G);
        pool.destroy();
        if (owner_stream) {
            cudaStreamSynchronize(owner_stream);
            cudaStreamDestroy(owner_stream);
        }
    }
};

namespace gahhg {

// Builds the exact index of one polygon on stream s (the caller's worker
// context); the grid borrows the stream and the scan state.
gahhg_status build_exact_grid(Polygon* P, int device, cudaStream_t s, void** scan, const gahhg_build_opts& base,
                              int top, int leaf, Grid** out)
{
    GAHHG_TRY(P->upload(s, device));
    Grid* g = new Grid();
    *out = g;
    g->poly = P;
    g->opts = base;
    g->opts.semantics = GAHHG_SEMANTICS_EXACT;
    if (top > 0) g->opts.lattice_top = top;
    if (leaf > 0) g->opts.lattice_leaf = leaf;
    g->device = device;
    g->stream = s;
    g->borrowed = true;
    g->scan_state = *scan;
    GAHHG_TRY(pool_alloc((void**)&g->d_err, sizeof(DeviceErrors), device, s));
    GAHHG_TRY(pool_alloc((void**)&g->d_counts, 64 * sizeof(int), device, s));
    GAHHG_CUDA_TRY(cudaMemsetAsync(g->d_err, 0, sizeof(DeviceErrors), s));
    const gahhg_status st = lattice_build(g);
    *scan = g->scan_state;  // the build may have grown it
    cudaFreeAsync(g->d_err, s);
    cudaFreeAsync(g->d_counts, s);
    g->d_err = nullptr;
    g->d_counts = nullptr;
    g->classified = true;
    return st;
}

// Builds the exact indexes of polys[0 .. count) together on stream s (a
// worker's context).
gahhg_status build_group(Polygon* const* polys, int count, int device, cudaStream_t s, void** scan,
                         const int* top, const int* leaf, GroupIndex** out)
{
    Grid g;
    g.device = device;
    g.stream = s;
    g.borrowed = true;
    g.scan_state = *scan;
    GAHHG_TRY(pool_alloc((void**)&g.d_err, sizeof(DeviceErrors), device, s));
    GAHHG_TRY(pool_alloc((void**)&g.d_counts, 64 * sizeof(int), device, s));
    GAHHG_CUDA_TRY(cudaMemsetAsync(g.d_err, 0, sizeof(DeviceErrors), s));
    const gahhg_status st = lattice_build_group(&g, polys, count, top, leaf, out);
    *scan = g.scan_state;  // the build may have grown it
    cudaFreeAsync(g.d_err, s);
    cudaFreeAsync(g.d_counts, s);
    g.d_err = nullptr;
    g.d_counts = nullptr;
    return st;
}

gahhg_status WorkerPool::create(int device, int n, int priority)
{
    this->device = device;
    streams.assign(n, nullptr);
    scans.assign(n, nullptr);
    for (int w = 0; w < n; w++) {
        if (cudaStreamCreateWithPriority(&streams[w], cudaStreamNonBlocking, priority) != cudaSuccess ||
            scan_state_reserve(&scans[w], 1u << 26) != GAHHG_OK) {
            set_error("worker stream or scan state creation failed");
            return GAHHG_ERR_CUDA;
        }
    }
    return GAHHG_OK;
}

void WorkerPool::destroy()
{
    for (size_t i = 0; i < streams.size(); i++) {
        if (scans[i]) scan_state_destroy(scans[i]);
        if (streams[i]) cudaStreamDestroy(streams[i]);
    }
    streams.clear();
    scans.clear();
}

// Builds grids[i] for every polygon with the pool's workers, one host thread
// per worker stream.  Returns the first failure (index in *failed).
gahhg_status WorkerPool::build_all(const std::vector<Polygon*>& polys, const gahhg_build_opts& base,
                                   const int* top, const int* leaf, std::vector<Grid*>& grids, int* failed)
{
    const int count = (int)polys.size();
    grids.assign(count, nullptr);
    std::atomic<int> next(0);
    std::atomic<int> bad(-1);
    std::mutex mu;
    std::string first_error;
    gahhg_status first_status = GAHHG_OK;
    auto worker = [&](int w) {
        cudaSetDevice(device);
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= count || bad.load() >= 0) break;
            const gahhg_status st = build_exact_grid(polys[i], device, streams[w], &scans[w], base,
                                                     top ? top[i] : 0, leaf ? leaf[i] : 0, &grids[i]);
            if (st != GAHHG_OK) {
                std::lock_guard<std::mutex> lock(mu);
                if (bad.load() < 0) {
                    bad.store(i);
                    first_status = st;
                    first_error = last_error();
                }
            }
        }
        cudaStreamSynchronize(streams[w]);
    };
    std::vector<std::thread> th;
    const int nw = std::min((int)streams.size(), std::max(count, 1));
    for (int w = 0; w < nw; w++) th.emplace_back(worker, w);
    for (auto& t : th) t.join();
    *failed = bad.load();
    if (*failed >= 0) set_error("polygon %d: %s", *failed, first_error.c_str());
    return *failed >= 0 ? first_status : GAHHG_OK;
}

}  // namespace gahhg

// Edges per group build: every step of a group runs once for all of its
// polygons, and its scratch grows with its edges (about 1 KB per edge at the
// peak of a C1-like build).
constexpr long long GROUP_EDGES = 1LL << 20;

extern "C" {

gahhg_status gahhg_batch_build(const gahhg_polygon* const* polys, int count, const gahhg_build_opts* opts,
                               const int* top_cells, const int* leaf_edges, int workers, gahhg_batch** out)
{
    if (!polys || count <= 0 || !out) {
        set_error("gahhg_batch_build: need at least one polygon");
        return GAHHG_ERR_ARG;
    }
    gahhg_build_opts base;
    if (opts)
        base = *opts;
    else
        gahhg_build_opts_init(&base);
    GAHHG_CUDA_TRY(cudaSetDevice(base.device));
    gahhg_batch* B = new gahhg_batch();
    B->device = base.device;
    B->count = count;
    B->polys.resize(count);
    B->grids.assign(count, nullptr);
    for (int i = 0; i < count; i++) {
        if (!polys[i]) {
            delete B;
            set_error("gahhg_batch_build: polygon %d is null", i);
            return GAHHG_ERR_ARG;
        }
        B->polys[i] = const_cast<Polygon*>(&polys[i]->p);
    }
    // group builds keep the GPU busy with a few workers; more only add scratch memory
    int nw = workers > 0 ? workers : (int)std::min(4u, std::max(1u, std::thread::hardware_concurrency()));
    nw = std::min(nw, count);
    if (B->pool.create(B->device, nw) != GAHHG_OK) {
        delete B;
        return GAHHG_ERR_CUDA;
    }
    const double t0 = now_seconds();
    // The workers' groups allocate and free their scratch concurrently: a
    // pool that trims its cache at every synchronisation would return it to
    // the driver and allocate it again, group after group.  Keep up to a
    // quarter of the device's memory cached (the pool then holds it until the
    // process exits or a later call lowers it).
    {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) GAHHG_TRY(pool_keep(B->device, total_b / 4));
    }
    // groups of consecutive polygons of at most GROUP_EDGES edges (a larger
    // polygon is a group of its own), built by the pool's workers
    std::vector<int> gstart(1, 0);
    {
        long long e = 0;
        for (int i = 0; i < count; i++) {
            const long long n = B->polys[i]->pv_num;
            if (i > gstart.back() && e + n > GROUP_EDGES) {
                gstart.push_back(i);
                e = 0;
            }
            e += n;
        }
        gstart.push_back(count);
    }
    const int ngroups = (int)gstart.size() - 1;
    B->groups.assign(ngroups, nullptr);
    {
        std::atomic<int> next(0), bad(-1);
        std::mutex mu;
        std::string first_error;
        gahhg_status first_status = GAHHG_OK;
        auto worker = [&](int w) {
            cudaSetDevice(B->device);
            for (;;) {
                const int k = next.fetch_add(1);
                if (k >= ngroups || bad.load() >= 0) break;
                const int i0 = gstart[k], i1 = gstart[k + 1];
                const gahhg_status st =
                    build_group(B->polys.data() + i0, i1 - i0, B->device, B->pool.streams[w], &B->pool.scans[w],
                                top_cells ? top_cells + i0 : nullptr, leaf_edges ? leaf_edges + i0 : nullptr,
                                &B->groups[k]);
                if (st != GAHHG_OK) {
                    std::lock_guard<std::mutex> lock(mu);
                    if (bad.load() < 0) {
                        bad.store(k);
                        first_status = st;
                        first_error = last_error();
                    }
                }
            }
            cudaStreamSynchronize(B->pool.streams[w]);
        };
        std::vector<std::thread> th;
        const int nt = std::min(nw, ngroups);
        for (int w = 0; w < nt; w++) th.emplace_back(worker, w);
        for (auto& t : th) t.join();
        if (bad.load() >= 0) {
            delete B;
            set_error("gahhg_batch_build: polygons %d..: %s", gstart[bad.load()], first_error.c_str());
            return first_status;
        }
    }
    // per-polygon query views, in one device table
    const size_t vb = lattice_view_bytes();
    std::vector<uint8_t> host(vb * count);
    long long bytes = 0, edges = 0;
    for (int k = 0; k < ngroups; k++) {
        bytes += group_bytes(B->groups[k]);
        for (int i = gstart[k]; i < gstart[k + 1]; i++) {
            group_view_write(B->groups[k], i - gstart[k], host.data() + vb * i);
            const long long sw = group_summary_words(B->groups[k], i - gstart[k]);
            B->swords.push_back((int)sw);
            edges += B->polys[i]->pv_num;
            if (sw > 4096) {
                delete B;
                set_error("gahhg_batch_build: polygon %d's summary exceeds the batch kernel's shared memory", i);
                return GAHHG_ERR_CAPACITY;
            }
        }
    }
    cudaStream_t s0 = B->pool.streams[0];
    GAHHG_TRY(B->views.reserve(host.size(), s0, false));
    GAHHG_CUDA_TRY(cudaMemcpyAsync(B->views.ptr, host.data(), host.size(), cudaMemcpyHostToDevice, s0));
    GAHHG_CUDA_TRY(cudaStreamSynchronize(s0));
    B->stats.build_s = now_seconds() - t0;
    B->stats.polygons = count;
    B->stats.edges = edges;
    B->stats.lattice_bytes = bytes;
    B->stats.workers = nw;
    *out = B;
    return GAHHG_OK;
}

int gahhg_batch_size(const gahhg_batch* b) { return b ? b->count : 0; }

// The captured query no longer matches the batch's settings: the next graph
// query captures again (an executable graph still running is freed when it
// completes).
static void drop_graph(gahhg_batch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
}

gahhg_status gahhg_batch_set_chunk(gahhg_batch* b, int chunk_points)
{
    if (!b || chunk_points < 256 || chunk_points > (1 << 20)) {
        set_error("chunk_points must be in [256, 1048576]");
        return GAHHG_ERR_ARG;
    }
    if (b->chunk_points != chunk_points) drop_graph(b);
    b->chunk_points = chunk_points;
    return GAHHG_OK;
}

gahhg_status gahhg_batch_shape_info(int shape, int* points_per_thread, int* blocks_per_sm)
{
    if (!batch_shape_info(shape, points_per_thread, blocks_per_sm)) {
        set_error("launch shape %d: there are %d shapes", shape, batch_shape_count());
        return GAHHG_ERR_ARG;
    }
    return GAHHG_OK;
}

gahhg_status gahhg_batch_set_shape(gahhg_batch* b, int shape)
{
    if (!b || !batch_shape_info(shape, nullptr, nullptr)) {
        set_error("launch shape must be in [0, %d)", batch_shape_count());
        return GAHHG_ERR_ARG;
    }
    if (b->shape != shape) drop_graph(b);
    b->shape = shape;
    return GAHHG_OK;
}

static gahhg_status check_offsets(const gahhg_batch* b, const int64_t* offsets)
{
    if (!offsets || offsets[0] != 0) {
        set_error("offsets must start at 0");
        return GAHHG_ERR_ARG;
    }
    for (int p = 0; p < b->count; p++)
        if (offsets[p + 1] < offsets[p]) {
            set_error("offsets must be non-decreasing");
            return GAHHG_ERR_ARG;
        }
    if (offsets[b->count] >= (int64_t)1 << 32) {
        set_error("a batch query takes fewer than 2^32 points");
        return GAHHG_ERR_CAPACITY;
    }
    return GAHHG_OK;
}

gahhg_status gahhg_batch_query_device(gahhg_batch* b, const double* d_lonlat, const int64_t* offsets,
                                      uint8_t* d_labels, int precision, void* stream, int sync)
{
    if (!b) return GAHHG_ERR_ARG;
    GAHHG_TRY(check_offsets(b, offsets));
    if (precision == GAHHG_QUERY_AUTO) precision = GAHHG_QUERY_FP32_FILTER;
    if (precision != GAHHG_QUERY_FP32_FILTER && precision != GAHHG_QUERY_FP64_FILTER) {
        set_error("batches answer with exact labels (FP32 or FP64 filter)");
        return GAHHG_ERR_ARG;
    }
    GAHHG_CUDA_TRY(cudaSetDevice(b->device));
    cudaStream_t s = (cudaStream_t)stream;
    const long long total = offsets[b->count];
    std::vector<uint8_t> chunks;
    int nchunks = 0;
    batch_make_chunks((const long long*)offsets, b->count, b->chunk_points, b->swords.data(), nullptr, chunks,
                      &nchunks);
    void* d_chunks = nullptr;
    uint32_t* queue = nullptr;
    unsigned int* counters = nullptr;
    uint64_t* d_stats = nullptr;
    GAHHG_TRY(pool_alloc(&d_chunks, std::max<size_t>(chunks.size(), 16), b->device, s));
    const long long qcap = std::max<long long>(total, 1);
    GAHHG_TRY(pool_alloc((void**)&queue, sizeof(uint32_t) * batch_queue_words(qcap), b->device, s));
    GAHHG_TRY(pool_alloc((void**)&counters, 8 * sizeof(unsigned int), b->device, s));
    if (!chunks.empty())
        GAHHG_CUDA_TRY(cudaMemcpyAsync(d_chunks, chunks.data(), chunks.size(), cudaMemcpyHostToDevice, s));
    if (sync) {
        GAHHG_TRY(pool_alloc((void**)&d_stats, 4 * sizeof(uint64_t), b->device, s));
        GAHHG_CUDA_TRY(cudaMemsetAsync(d_stats, 0, 4 * sizeof(uint64_t), s));
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (sync) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, s);
    }
    gahhg_status st = batch_query_launch(b->views.ptr, d_chunks, nchunks, d_lonlat, d_labels, precision, queue,
                                         qcap, counters, d_stats, s, b->device, true, b->shape);
    if (sync && st == GAHHG_OK) {
        cudaEventRecord(e1, s);
        uint64_t c[4] = {0, 0, 0, 0};
        cudaMemcpyAsync(c, d_stats, sizeof(c), cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) {
            set_error("batch query failed: %s", cudaGetErrorString(cudaGetLastError()));
            st = GAHHG_ERR_CUDA;
        } else {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            b->stats.query_s = ms * 1e-3;
            b->stats.query_points = total;
            b->stats.esc_fp64 = (long long)c[0];
            b->stats.esc_exact = (long long)c[1];
            b->stats.boundary_points = (long long)c[2];
            b->stats.in_count = (long long)c[3];
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFreeAsync(d_chunks, s);
    cudaFreeAsync(queue, s);
    cudaFreeAsync(counters, s);
    if (d_stats) cudaFreeAsync(d_stats, s);
    return st;
}

gahhg_status gahhg_batch_query_graph(gahhg_batch* b, const double* d_lonlat, const int64_t* offsets,
                                     uint8_t* d_labels, int precision, void* stream)
{
    if (!b) return GAHHG_ERR_ARG;
    GAHHG_TRY(check_offsets(b, offsets));
    if (precision == GAHHG_QUERY_AUTO) precision = GAHHG_QUERY_FP32_FILTER;
    if (precision != GAHHG_QUERY_FP32_FILTER && precision != GAHHG_QUERY_FP64_FILTER) {
        set_error("batches answer with exact labels (FP32 or FP64 filter)");
        return GAHHG_ERR_ARG;
    }
    GAHHG_CUDA_TRY(cudaSetDevice(b->device));
    cudaStream_t s = (cudaStream_t)stream;
    const bool same = b->exec && b->g_lonlat == d_lonlat && b->g_labels == d_labels && b->g_precision == precision &&
                      b->g_offsets.size() == (size_t)b->count + 1 &&
                      std::equal(b->g_offsets.begin(), b->g_offsets.end(), offsets);
    if (!same) {
        // (re)build the workspace and capture the launch sequence once
        if (b->exec) {
            cudaGraphExecDestroy(b->exec);
            b->exec = nullptr;
        }
        if (!b->owner_stream) GAHHG_CUDA_TRY(cudaStreamCreateWithFlags(&b->owner_stream, cudaStreamNonBlocking));
        cudaStream_t ws = b->owner_stream;
        const long long total = offsets[b->count];
        std::vector<uint8_t> chunks;
        batch_make_chunks((const long long*)offsets, b->count, b->chunk_points, b->swords.data(), nullptr, chunks,
                          &b->g_nchunks);
        GAHHG_TRY(b->g_chunks.reserve(std::max<size_t>(chunks.size(), 16), ws, false));
        b->g_qcap = std::max<long long>(total, 1);
        GAHHG_TRY(b->g_queue.reserve(batch_queue_words(b->g_qcap), ws, false));
        GAHHG_TRY(b->g_counters.reserve(8, ws, false));
        if (!chunks.empty())
            GAHHG_CUDA_TRY(cudaMemcpyAsync(b->g_chunks.ptr, chunks.data(), chunks.size(), cudaMemcpyHostToDevice, ws));
        GAHHG_CUDA_TRY(cudaStreamSynchronize(ws));
        cudaStream_t cs = nullptr;
        GAHHG_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t graph = nullptr;
        gahhg_status st = GAHHG_OK;
        if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            st = GAHHG_ERR_CUDA;
        } else {
            st = batch_query_launch(b->views.ptr, b->g_chunks.ptr, b->g_nchunks, d_lonlat, d_labels, precision,
                                    b->g_queue.ptr, b->g_qcap, b->g_counters.ptr, nullptr, cs, b->device, true,
                                    b->shape);
            if (cudaStreamEndCapture(cs, &graph) != cudaSuccess) st = GAHHG_ERR_CUDA;
        }
        cudaStreamDestroy(cs);
        if (st != GAHHG_OK || !graph) {
            if (graph) cudaGraphDestroy(graph);
            set_error("batch graph capture failed: %s", cudaGetErrorString(cudaGetLastError()));
            return GAHHG_ERR_CUDA;
        }
        cudaError_t e = cudaGraphInstantiate(&b->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            b->exec = nullptr;
            set_error("cudaGraphInstantiate: %s", cudaGetErrorString(e));
            return GAHHG_ERR_CUDA;
        }
        b->g_lonlat = d_lonlat;
        b->g_labels = d_labels;
        b->g_precision = precision;
        b->g_offsets.assign(offsets, offsets + b->count + 1);
    }
    GAHHG_CUDA_TRY(cudaGraphLaunch(b->exec, s));
    return GAHHG_OK;
}

gahhg_status gahhg_batch_stats_get(const gahhg_batch* b, gahhg_batch_stats* s)
{
    if (!b || !s) return GAHHG_ERR_ARG;
    *s = b->stats;
    return GAHHG_OK;
}

void gahhg_batch_free(gahhg_batch* b) { delete b; }

}  // extern "C"
