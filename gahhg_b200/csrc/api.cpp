// api.cpp - the C ABI (include/gahhg.h) over the host objects.
#include <atomic>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <mutex>

#include "gahhg_internal.h"

namespace gahhg {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

const char* last_error() { return g_err; }

static std::mutex g_pool_mu;
static cudaMemPool_t g_pools[64] = {};
// set once per device under g_pool_mu; read without the lock afterwards
// (every allocation of every build worker asks for its device's pool)
static std::atomic<cudaMemPool_t> g_pool_ready[64] = {};

static gahhg_status device_pool(int device, cudaMemPool_t* out)
{
    if (device < 0 || device >= 64) {
        set_error("device ordinal %d out of range", device);
        return GAHHG_ERR_ARG;
    }
    if (cudaMemPool_t p = g_pool_ready[device].load(std::memory_order_acquire)) {
        *out = p;
        return GAHHG_OK;
    }
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pools[device]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        GAHHG_CUDA_TRY(cudaMemPoolCreate(&g_pools[device], &props));
        uint64_t keep = 4ull << 30;  // keep up to 4 GB cached between calls
        GAHHG_CUDA_TRY(cudaMemPoolSetAttribute(g_pools[device], cudaMemPoolAttrReleaseThreshold, &keep));
        g_pool_ready[device].store(g_pools[device], std::memory_order_release);
    }
    *out = g_pools[device];
    return GAHHG_OK;
}

gahhg_status pool_alloc(void** p, size_t bytes, int device, cudaStream_t s)
{
    cudaMemPool_t pool;
    GAHHG_TRY(device_pool(device, &pool));
    GAHHG_CUDA_TRY(cudaMallocFromPoolAsync(p, bytes, pool, s));
    return GAHHG_OK;
}

gahhg_status pool_keep(int device, size_t bytes)
{
    cudaMemPool_t pool;
    GAHHG_TRY(device_pool(device, &pool));
    std::lock_guard<std::mutex> lock(g_pool_mu);
    uint64_t cur = 0;
    GAHHG_CUDA_TRY(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &cur));
    if ((uint64_t)bytes > cur) {
        uint64_t v = bytes;
        GAHHG_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &v));
    }
    return GAHHG_OK;
}

double now_seconds()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

gahhg_status Polygon::upload(cudaStream_t s, int device)
{
    if (d_pv) return GAHHG_OK;
    if (pv_num <= 0) {
        set_error("polygon has no edges");
        return GAHHG_ERR_ARG;
    }
    if (s) {
        // stream-ordered from the library pool: neither the upload nor the
        // release synchronises other streams
        GAHHG_TRY(pool_alloc((void**)&d_pv, sizeof(D3) * pv_num, device, s));
        GAHHG_TRY(pool_alloc((void**)&d_pe, sizeof(int) * 2 * pv_num, device, s));
        pooled = true;
        GAHHG_CUDA_TRY(cudaMemcpyAsync(d_pv, pv.data(), sizeof(D3) * pv_num, cudaMemcpyHostToDevice, s));
        GAHHG_CUDA_TRY(cudaMemcpyAsync(d_pe, pe.data(), sizeof(int) * 2 * pv_num, cudaMemcpyHostToDevice, s));
        return GAHHG_OK;
    }
    GAHHG_CUDA_TRY(cudaMalloc(&d_pv, sizeof(D3) * pv_num));
    GAHHG_CUDA_TRY(cudaMalloc(&d_pe, sizeof(int) * 2 * pv_num));
    GAHHG_CUDA_TRY(cudaMemcpy(d_pv, pv.data(), sizeof(D3) * pv_num, cudaMemcpyHostToDevice));
    GAHHG_CUDA_TRY(cudaMemcpy(d_pe, pe.data(), sizeof(int) * 2 * pv_num, cudaMemcpyHostToDevice));
    return GAHHG_OK;
}

void Polygon::copy_host(const Polygon& o)
{
    pv_num = o.pv_num;
    num_rings = o.num_rings;
    lonlat = o.lonlat;
    pv = o.pv;
    pe = o.pe;
    ring_start = o.ring_start;
    path = o.path;
}

Polygon::~Polygon()
{
    // pooled copies were last used by kernels whose completion the owner has
    // observed; the legacy stream does not wait for non-blocking streams
    if (pooled) {
        if (d_pv) cudaFreeAsync(d_pv, 0);
        if (d_pe) cudaFreeAsync(d_pe, 0);
        return;
    }
    if (d_pv) cudaFree(d_pv);
    if (d_pe) cudaFree(d_pe);
}

void free_query_layout(void* p);
size_t query_layout_bytes(const void* p);
void scan_state_destroy(void* state);

Grid::~Grid()
{
    V.release();
    B.release();
    C.release();
    refs.release();
    cell_a.release();
    cell_b.release();
    off_a.release();
    off_b.release();
    edge_cur.release();
    edge_prev.release();
    edge_cnt.release();
    edge_off.release();
    ref_cell.release();
    ref_flag.release();
    ref_edge.release();
    type_old.release();
    type_cur.release();
    type_next.release();
    if (d_err) cudaFree(d_err);
    if (d_counts) cudaFree(d_counts);
    if (h_counts) cudaFreeHost(h_counts);
    free_query_layout(qlayout);
    lattice_free(lattice);
    if (aux_stream) cudaStreamDestroy(aux_stream);
    if (!borrowed) {
        scan_state_destroy(scan_state);
        if (stream) cudaStreamDestroy(stream);
    }
}

static void fill_stats(Grid* g)
{
    gahhg_stats& s = g->stats;
    s.pv_num = g->poly->pv_num;
    s.lattice_bytes = (long long)lattice_bytes(g->lattice);
    if (!g->hierarchy) return;
    const Level& L = g->levels[g->gnum - 1];
    s.depth = g->gnum;
    s.pv_num = g->poly->pv_num;
    s.vnum = L.vstart + L.vnum;
    s.bnum = L.bstart + L.bnum;
    s.cnum = L.cstart + L.cnum;
    s.rnum = L.rnum;
    // sizeof(GAHHG) + sizeof(GAHHGGrid)*gnum + sizeof(GPISPParam) + sizeof(GPISPStat)
    // on x64 (source/GPISPAHHG.cu:2100): 144 + 28*gnum + 552 + 96
    s.cpu_space = 792 + 28 * g->gnum;
    s.gpu_min_space = 24 * s.vnum + 48 * s.bnum + 28 * s.cnum + 4 * s.rnum;
    s.gamma = g->gamma;
}

// The hexagon hierarchy of an exact grid, built (and classified, when the
// grid was) the first time something needs it; exact queries never do.
static gahhg_status ensure_hierarchy(Grid* g)
{
    std::lock_guard<std::mutex> lock(g->hierarchy_mu);
    if (g->hierarchy) return GAHHG_OK;
    GAHHG_CUDA_TRY(cudaSetDevice(g->device));
    GAHHG_TRY(grid_build(g));
    g->hierarchy = true;
    if (g->classified) {
        GAHHG_TRY(grid_classify(g));
        GAHHG_TRY(grid_prepare_query(g));
    }
    fill_stats(g);
    return GAHHG_OK;
}

// process-wide knobs (gahhg_set_knob)
namespace {
constexpr int KNOB_COUNT = 8;
constexpr long long KNOB_DEFAULT[KNOB_COUNT] = {0, 0, 1 << 16, 1 << 22, 1 << 20, 0, 0, 0};  // index = gahhg_knob
std::atomic<long long> g_knobs[KNOB_COUNT] = {0, 0, 1 << 16, 1 << 22, 1 << 20, 0, 0, 0};
// knobs that choose among a few modes (0 .. knob_modes - 1) rather than limits
inline int knob_modes(int k) { return k == GAHHG_KNOB_GROUPED_PASS2 ? 4 : 0; }
}  // namespace

long long knob(int k) { return (k > 0 && k < KNOB_COUNT) ? g_knobs[k].load(std::memory_order_relaxed) : 0; }

}  // namespace gahhg

using namespace gahhg;

extern "C" {

void gahhg_build_opts_init(gahhg_build_opts* o)
{
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->max_depth = 15;
    o->auto_depth = 1;
    o->semantics = GAHHG_SEMANTICS_EXACT;
    o->lattice_top = 0;
    o->lattice_leaf = 0;
    o->device = 0;
    o->verbose = 0;
}

const char* gahhg_last_error(void) { return last_error(); }
int gahhg_abi_version(void) { return GAHHG_ABI_VERSION; }

gahhg_status gahhg_set_knob(int k, long long value)
{
    if (k < GAHHG_KNOB_GROUPED_PASS2 || k > GAHHG_KNOB_STAGING_POLL_LIMIT) {
        set_error("unknown knob %d", k);
        return GAHHG_ERR_ARG;
    }
    const int modes = knob_modes(k);
    if (modes ? (value < 0 || value >= modes) : (value < 0 || value > KNOB_DEFAULT[k])) {
        if (modes)
            set_error("knob %d takes 0 .. %d, not %lld", k, modes - 1, value);
        else
            set_error("knob %d takes 0 .. its default, not %lld", k, value);
        return GAHHG_ERR_ARG;
    }
    gahhg::g_knobs[k].store(value, std::memory_order_relaxed);
    return GAHHG_OK;
}

long long gahhg_get_knob(int k) { return gahhg::knob(k); }

gahhg_status gahhg_staging_fallbacks(int device, unsigned long long* count)
{
    if (!count) {
        set_error("null count");
        return GAHHG_ERR_ARG;
    }
    return lattice_staging_fallbacks(device, count);
}

gahhg_status gahhg_polygon_load(const char* path, gahhg_polygon** out)
{
    if (!path || !out) return GAHHG_ERR_ARG;
    gahhg_polygon* p = new gahhg_polygon();
    gahhg_status s = load_polygon_file(path, &p->p);
    if (s != GAHHG_OK) {
        delete p;
        return s;
    }
    *out = p;
    return GAHHG_OK;
}

gahhg_status gahhg_polygon_from_rings(const double* lonlat, const int64_t* ring_offsets, int nrings,
                                      gahhg_polygon** out)
{
    if (!out) return GAHHG_ERR_ARG;
    gahhg_polygon* p = new gahhg_polygon();
    gahhg_status s = polygon_from_rings(lonlat, ring_offsets, nrings, &p->p);
    if (s != GAHHG_OK) {
        delete p;
        return s;
    }
    *out = p;
    return GAHHG_OK;
}

int gahhg_polygon_num_edges(const gahhg_polygon* p) { return p ? p->p.pv_num : 0; }

gahhg_status gahhg_polygon_export(const gahhg_polygon* p, double* xyz, int* pe)
{
    if (!p) return GAHHG_ERR_ARG;
    if (xyz) memcpy(xyz, p->p.pv.data(), sizeof(D3) * p->p.pv_num);
    if (pe) memcpy(pe, p->p.pe.data(), sizeof(int) * 2 * p->p.pv_num);
    return GAHHG_OK;
}

void gahhg_polygon_free(gahhg_polygon* p) { delete p; }

gahhg_status gahhg_points_load(const char* path, gahhg_points** out)
{
    if (!path || !out) return GAHHG_ERR_ARG;
    gahhg_points* p = new gahhg_points();
    gahhg_status s = load_points_file(path, &p->p);
    if (s != GAHHG_OK) {
        delete p;
        return s;
    }
    *out = p;
    return GAHHG_OK;
}

size_t gahhg_points_count(const gahhg_points* p) { return p ? p->p.n : 0; }
const double* gahhg_points_lonlat(const gahhg_points* p) { return p ? p->p.lonlat.get() : nullptr; }

gahhg_status gahhg_points_load_ex(const char* path, int flags, gahhg_points** out)
{
    if (!path || !out) return GAHHG_ERR_ARG;
    gahhg_points* p = new gahhg_points();
    if ((flags & GAHHG_POINTS_USE_SIDECAR) && load_points_sidecar(path, &p->p) == GAHHG_OK) {
        *out = p;
        return GAHHG_OK;
    }
    gahhg_status s = load_points_file(path, &p->p);
    if (s == GAHHG_OK && (flags & GAHHG_POINTS_WRITE_SIDECAR)) s = write_points_sidecar(path, p->p);
    if (s != GAHHG_OK) {
        delete p;
        return s;
    }
    *out = p;
    return GAHHG_OK;
}
void gahhg_points_free(gahhg_points* p) { delete p; }

gahhg_status gahhg_build(const gahhg_polygon* poly, const gahhg_build_opts* opts, gahhg_grid** out)
{
    if (!poly || !out) {
        set_error("gahhg_build: null argument");
        return GAHHG_ERR_ARG;
    }
    gahhg_build_opts o;
    if (opts)
        o = *opts;
    else
        gahhg_build_opts_init(&o);
    if (o.max_depth < 1 || o.max_depth > 30) {
        set_error("max_depth must be in [1, 30]");
        return GAHHG_ERR_ARG;
    }
    GAHHG_CUDA_TRY(cudaSetDevice(o.device));
    gahhg_polygon* mp = const_cast<gahhg_polygon*>(poly);
    GAHHG_TRY(mp->p.upload());
    gahhg_grid* G = new gahhg_grid();
    Grid* g = &G->g;
    g->poly = &poly->p;
    g->opts = o;
    g->device = o.device;
    cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        set_error("cudaStreamCreate: %s", cudaGetErrorString(e));
        delete G;
        return GAHHG_ERR_CUDA;
    }
    gahhg_status s = GAHHG_OK;
    if (o.semantics == GAHHG_SEMANTICS_EXACT) {
        // the exact index alone: the hierarchy waits until something needs it
        const double t0 = now_seconds();
        s = grid_alloc_common(g);
        if (s == GAHHG_OK) s = lattice_build(g);
        g->stats.lattice_s = now_seconds() - t0;
    } else {
        s = grid_build(g);
        g->hierarchy = s == GAHHG_OK;
    }
    if (s != GAHHG_OK) {
        delete G;
        return s;
    }
    fill_stats(g);
    *out = G;
    return GAHHG_OK;
}

gahhg_status gahhg_classify(gahhg_grid* G)
{
    if (!G) return GAHHG_ERR_ARG;
    GAHHG_CUDA_TRY(cudaSetDevice(G->g.device));
    {
        std::lock_guard<std::mutex> lock(G->g.hierarchy_mu);
        if (G->g.hierarchy) {
            GAHHG_TRY(grid_classify(&G->g));
            GAHHG_TRY(grid_prepare_query(&G->g));
        }
        G->g.classified = true;  // an exact grid without its hierarchy is query-ready
    }
    fill_stats(&G->g);
    return GAHHG_OK;
}

void gahhg_grid_free(gahhg_grid* G)
{
    if (!G) return;
    cudaSetDevice(G->g.device);
    delete G;
}

static gahhg_status run_query(Grid* g, const double* d_lonlat, size_t n, uint8_t* d_labels, int precision,
                              cudaStream_t s, uint64_t* d_counters)
{
    if (!g->classified) {
        set_error("query before classify");
        return GAHHG_ERR_STATE;
    }
    if (precision == GAHHG_QUERY_AUTO)
        precision = g->lattice ? GAHHG_QUERY_FP32_FILTER : GAHHG_QUERY_REFERENCE_FP64;
    if (precision == GAHHG_QUERY_REFERENCE_FP64) {
        GAHHG_TRY(ensure_hierarchy(g));
        return grid_query_ref(g, d_lonlat, n, d_labels, s, d_counters);
    }
    if (precision == GAHHG_QUERY_FP32_FILTER || precision == GAHHG_QUERY_FP64_FILTER) {
        if (!g->lattice) {
            set_error("exact precision needs a grid built with GAHHG_SEMANTICS_EXACT");
            return GAHHG_ERR_STATE;
        }
        if ((uintptr_t)d_lonlat & 15u) {
            set_error("exact queries read lon/lat in 16-byte units: the device buffer must be 16-byte aligned");
            return GAHHG_ERR_ARG;
        }
        return lattice_query(g, d_lonlat, n, d_labels, precision, s, d_counters);
    }
    set_error("unknown precision %d", precision);
    return GAHHG_ERR_ARG;
}

gahhg_status gahhg_query_device(gahhg_grid* G, const double* d_lonlat, size_t n, uint8_t* d_labels, int precision,
                                void* stream, int sync)
{
    if (!G || (n && (!d_lonlat || !d_labels))) return GAHHG_ERR_ARG;
    Grid* g = &G->g;
    cudaStream_t s = (cudaStream_t)stream;
    if (!sync) return run_query(g, d_lonlat, n, d_labels, precision, s, nullptr);
    uint64_t* d_cnt = nullptr;
    GAHHG_TRY(pool_alloc((void**)&d_cnt, 4 * sizeof(uint64_t), g->device, s));
    GAHHG_CUDA_TRY(cudaMemsetAsync(d_cnt, 0, 4 * sizeof(uint64_t), s));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    gahhg_status st = run_query(g, d_lonlat, n, d_labels, precision, s, d_cnt);
    cudaEventRecord(e1, s);
    uint64_t cnt[4] = {0, 0, 0, 0};
    if (st == GAHHG_OK) {
        cudaMemcpyAsync(cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            set_error("query: %s", cudaGetErrorString(e));
            st = GAHHG_ERR_CUDA;
        }
    }
    float ms = 0.f;
    if (st == GAHHG_OK) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(d_cnt, s);
    if (st != GAHHG_OK) return st;
    g->stats.query_s = ms * 1e-3;
    g->stats.query_points = (long long)n;
    g->stats.esc_fp64 = (long long)cnt[0];
    g->stats.esc_exact = (long long)cnt[1];
    g->stats.boundary_points = (long long)cnt[2];
    g->stats.in_count = (long long)cnt[3];
    return GAHHG_OK;
}

gahhg_status gahhg_query_device_noalloc(gahhg_grid* G, const double* d_lonlat, size_t n, uint8_t* d_labels,
                                        int precision, void* stream)
{
    if (!G || (n && (!d_lonlat || !d_labels))) {
        set_error("gahhg_query_device_noalloc: null argument");
        return GAHHG_ERR_ARG;
    }
    Grid* g = &G->g;
    if (!g->classified) {
        set_error("query before classify");
        return GAHHG_ERR_STATE;
    }
    if (!g->lattice) {
        set_error("gahhg_query_device_noalloc needs a grid built with GAHHG_SEMANTICS_EXACT");
        return GAHHG_ERR_STATE;
    }
    if (precision == GAHHG_QUERY_AUTO) precision = GAHHG_QUERY_FP32_FILTER;
    if (precision != GAHHG_QUERY_FP32_FILTER && precision != GAHHG_QUERY_FP64_FILTER) {
        set_error("gahhg_query_device_noalloc supports the exact precisions only");
        return GAHHG_ERR_ARG;
    }
    GAHHG_CUDA_TRY(cudaSetDevice(g->device));
    return lattice_query_noalloc(g, d_lonlat, n, d_labels, precision, (cudaStream_t)stream);
}

long long gahhg_query_noalloc_max_points(void) { return lattice_noalloc_max_points(); }

// Host buffers: chunks of E2E_CHUNK points alternate between the grid's
// stream and an auxiliary one, each chunk copied in, queried and copied out
// on its stream, so one chunk's host-to-device copy overlaps the previous
// chunk's query and device-to-host copy (the copy engines run both
// directions at once).  Device memory: two chunk buffers.  query_s sums the
// device time of the query launches alone, like the reference's PISPTime.
static constexpr size_t E2E_CHUNK = (size_t)1 << 23;

gahhg_status gahhg_query(gahhg_grid* G, const double* lonlat, size_t n, uint8_t* labels, int precision)
{
    if (!G || (n && (!lonlat || !labels))) return GAHHG_ERR_ARG;
    Grid* g = &G->g;
    if (!g->classified) {
        set_error("query before classify");
        return GAHHG_ERR_STATE;
    }
    GAHHG_CUDA_TRY(cudaSetDevice(g->device));
    if (n == 0) return GAHHG_OK;
    if (!g->aux_stream) GAHHG_CUDA_TRY(cudaStreamCreateWithFlags(&g->aux_stream, cudaStreamNonBlocking));
    cudaStream_t st[2] = {g->stream, g->aux_stream};
    const size_t chunk = std::min(n, E2E_CHUNK);
    const size_t nchunks = (n + chunk - 1) / chunk;
    uint8_t* buf[2] = {nullptr, nullptr};
    uint64_t* d_cnt = nullptr;
    GAHHG_TRY(pool_alloc((void**)&d_cnt, 4 * sizeof(uint64_t), g->device, st[0]));
    GAHHG_CUDA_TRY(cudaMemsetAsync(d_cnt, 0, 4 * sizeof(uint64_t), st[0]));
    std::vector<cudaEvent_t> ev(2 * nchunks + 2, nullptr);
    for (auto& e : ev) cudaEventCreate(&e);
    // the auxiliary stream starts after the counters are cleared
    cudaEventRecord(ev[2 * nchunks], st[0]);
    cudaStreamWaitEvent(st[1], ev[2 * nchunks], 0);
    gahhg_status rc = GAHHG_OK;
    for (int b = 0; b < 2 && rc == GAHHG_OK && (size_t)b < nchunks; b++)
        rc = pool_alloc((void**)&buf[b], chunk * 17, g->device, st[b]);
    for (size_t k = 0; k < nchunks && rc == GAHHG_OK; k++) {
        const int b = (int)(k & 1);
        cudaStream_t s = st[b];
        const size_t off = k * chunk, m = std::min(chunk, n - off);
        double* d_ll = (double*)buf[b];
        uint8_t* d_lab = buf[b] + chunk * 16;
        if (cudaMemcpyAsync(d_ll, lonlat + 2 * off, m * 16, cudaMemcpyHostToDevice, s) != cudaSuccess) {
            set_error("query copy-in: %s", cudaGetErrorString(cudaGetLastError()));
            rc = GAHHG_ERR_CUDA;
            break;
        }
        cudaEventRecord(ev[2 * k], s);
        rc = run_query(g, d_ll, m, d_lab, precision, s, d_cnt);
        cudaEventRecord(ev[2 * k + 1], s);
        if (rc == GAHHG_OK && cudaMemcpyAsync(labels + off, d_lab, m, cudaMemcpyDeviceToHost, s) != cudaSuccess) {
            set_error("query copy-out: %s", cudaGetErrorString(cudaGetLastError()));
            rc = GAHHG_ERR_CUDA;
        }
    }
    // join the auxiliary stream, then read the counters
    cudaEventRecord(ev[2 * nchunks + 1], st[1]);
    cudaStreamWaitEvent(st[0], ev[2 * nchunks + 1], 0);
    uint64_t cnt[4] = {0, 0, 0, 0};
    cudaMemcpyAsync(cnt, d_cnt, sizeof(cnt), cudaMemcpyDeviceToHost, st[0]);
    const cudaError_t e = cudaStreamSynchronize(st[0]);
    if (rc == GAHHG_OK && e != cudaSuccess) {
        set_error("query: %s", cudaGetErrorString(e));
        rc = GAHHG_ERR_CUDA;
    }
    if (rc == GAHHG_OK) {
        double ms_total = 0.0;
        for (size_t k = 0; k < nchunks; k++) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[2 * k], ev[2 * k + 1]);
            ms_total += ms;
        }
        g->stats.query_s = ms_total * 1e-3;
        g->stats.query_points = (long long)n;
        g->stats.esc_fp64 = (long long)cnt[0];
        g->stats.esc_exact = (long long)cnt[1];
        g->stats.boundary_points = (long long)cnt[2];
        g->stats.in_count = (long long)cnt[3];
    }
    for (int b = 0; b < 2; b++)
        if (buf[b]) cudaFreeAsync(buf[b], st[0]);
    cudaFreeAsync(d_cnt, st[0]);
    cudaStreamSynchronize(st[0]);
    for (auto& x : ev) cudaEventDestroy(x);
    return rc;
}

gahhg_status gahhg_stats_get(const gahhg_grid* G, gahhg_stats* s)
{
    if (!G || !s) return GAHHG_ERR_ARG;
    *s = G->g.stats;
    return GAHHG_OK;
}

int gahhg_grid_depth(const gahhg_grid* G)
{
    if (!G || ensure_hierarchy(const_cast<Grid*>(&G->g)) != GAHHG_OK) return 0;
    return G->g.gnum;
}

gahhg_status gahhg_grid_export(const gahhg_grid* G, int* levels, double* v, void* b, void* c, int* refs)
{
    if (!G) return GAHHG_ERR_ARG;
    GAHHG_TRY(ensure_hierarchy(const_cast<Grid*>(&G->g)));
    const Grid* g = &G->g;
    const Level& L = g->levels[g->gnum - 1];
    GAHHG_CUDA_TRY(cudaSetDevice(g->device));
    if (levels) memcpy(levels, g->levels.data(), sizeof(Level) * g->gnum);
    if (v) GAHHG_CUDA_TRY(cudaMemcpy(v, g->V.ptr, sizeof(D3) * (L.vstart + L.vnum), cudaMemcpyDeviceToHost));
    if (b) GAHHG_CUDA_TRY(cudaMemcpy(b, g->B.ptr, sizeof(Border) * (L.bstart + L.bnum), cudaMemcpyDeviceToHost));
    if (c) GAHHG_CUDA_TRY(cudaMemcpy(c, g->C.ptr, sizeof(Cell) * (L.cstart + L.cnum), cudaMemcpyDeviceToHost));
    if (refs && L.rnum) GAHHG_CUDA_TRY(cudaMemcpy(refs, g->refs.ptr, sizeof(int) * L.rnum, cudaMemcpyDeviceToHost));
    return GAHHG_OK;
}

gahhg_status gahhg_grid0_export(double* v, void* b, void* c)
{
    std::vector<D3> V;
    std::vector<Border> B;
    std::vector<Cell> C;
    build_grid0(V, B, C);
    if (v) memcpy(v, V.data(), sizeof(D3) * V.size());
    if (b) memcpy(b, B.data(), sizeof(Border) * B.size());
    if (c) memcpy(c, C.data(), sizeof(Cell) * C.size());
    return GAHHG_OK;
}

gahhg_status gahhg_report_append(const gahhg_grid* G, const char* polyfile, const char* tpfile, long long npoints,
                                 const char* path, int dest_stdout)
{
    if (!G) return GAHHG_ERR_ARG;
    GAHHG_TRY(ensure_hierarchy(const_cast<Grid*>(&G->g)));
    const gahhg_stats& s = G->g.stats;
    FILE* fp = stdout;
    if (!dest_stdout) {
        fp = fopen(path, "a");
        if (!fp) {
            printf("Can not open file %s\n.", path);
            set_error("cannot open %s", path);
            return GAHHG_ERR_IO;
        }
    }
    // GPISP::exportStat2TXT (source/GPISPAHHG.cu:2115-2161)
    time_t now = time(nullptr);
    struct tm lt;
    localtime_r(&now, &lt);
    fprintf(fp, "\n----------------------------------------%d/%d/%d %d:%d:%d-----------------------------------------\n",
            lt.tm_year + 1900, lt.tm_mon + 1, lt.tm_mday, lt.tm_hour, lt.tm_min, lt.tm_sec);
    fprintf(fp, "\nPolygon file: %s\n", polyfile);
    fprintf(fp, "Number of polygon vertice: %d\n", s.pv_num);
    fprintf(fp, "Query point file: %s\n", tpfile);
    fprintf(fp, "Number of query points: %d\n", (int)npoints);
    fprintf(fp, "Depth of GAHHG: %d\n", s.depth);
    fprintf(fp, "Time of preprocessing: %f seconds (creat GAHHG: %f seconds, classify GAHHG: %f seconds)\n",
            s.pre_s, s.create_s, s.classify_s);
    fprintf(fp, "Storage overhead of GAHHG on CPU: %d Bytes\n", s.cpu_space);
    fprintf(fp, "Storage overhead of GAHHG on GPU: %d KB\n", (int)(s.gpu_min_space / 1000));
    fprintf(fp, "Total test time for all query points: %f seconds\n", s.query_s);
    fprintf(fp, "Average test time per query point: %.5e seconds\n", npoints ? s.query_s / npoints : 0.0);
    fprintf(fp, "Test result: inside %d, outside %d\n", (int)s.in_count, (int)(npoints - s.in_count));
    fprintf(fp, "\n---------------------------------------------------------------------------------------------------\n");
    if (!dest_stdout) fclose(fp);
    return GAHHG_OK;
}

gahhg_status gahhg_result_write(const char* path, const uint8_t* labels, size_t n)
{
    FILE* fp = fopen(path, "w");
    if (!fp) {
        printf("Can not open file %s\n.", path);
        set_error("cannot open %s", path);
        return GAHHG_ERR_IO;
    }
    // one "1\n" or "0\n" per point (source/GPISPTP.cu:92-96), written in blocks
    std::vector<char> buf;
    buf.reserve(1 << 20);
    for (size_t i = 0; i < n; i++) {
        buf.push_back(labels[i] == CELL_IN ? '1' : '0');
        buf.push_back('\n');
        if (buf.size() >= (1 << 20)) {
            fwrite(buf.data(), 1, buf.size(), fp);
            buf.clear();
        }
    }
    if (!buf.empty()) fwrite(buf.data(), 1, buf.size(), fp);
    fclose(fp);
    return GAHHG_OK;
}

}  // extern "C"
