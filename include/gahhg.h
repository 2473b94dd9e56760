/*
 * gahhg.h - C ABI of the B200 point-in-spherical-polygon engine.
 *
 * Drop-in for the build -> classify -> query path of GAHHG.  Each entry point
 * names the reference interface it replaces (paths relative to the GAHHG
 * repository).  Plain pointers and sizes only; `stream` is a cudaStream_t
 * passed as void* (NULL = the legacy default stream).
 *
 * Labels are one byte per point with the reference's cell codes
 * (source/GPISPParam.h:9-11): 0 = undefined, 1 = outside, 2 = inside.  The
 * result CSV prints "1" for 2 and "0" otherwise (source/GPISPTP.cu:92-96).
 *
 * Two label semantics:
 *   GAHHG_SEMANTICS_REFERENCE  the reference's epsilon rules, FP64, bit for bit
 *                              (points within ~1e-8 rad of an edge follow the
 *                              reference's tolerance tests);
 *   GAHHG_SEMANTICS_EXACT      the exact sign of the orientation determinants
 *                              on the canonical FP64 XYZ (gahhg_canon.h), with
 *                              symbolic perturbation for exact zeros.
 * Every call returns a status; gahhg_last_error() holds the message of the
 * last failure on the calling thread.
 */
#ifndef GAHHG_H
#define GAHHG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GAHHG_ABI_VERSION 1

typedef enum {
    GAHHG_OK = 0,
    GAHHG_ERR_IO = -1,        /* file cannot be opened (reference returns -1) */
    GAHHG_ERR_FORMAT = -2,    /* malformed POLYGON / CSV content (reference returns -1) */
    GAHHG_ERR_ARG = -3,       /* invalid argument */
    GAHHG_ERR_CUDA = -4,      /* CUDA runtime error */
    GAHHG_ERR_DEVICE = -5,    /* a kernel reported a bounded failure (walk limit, bad index) */
    GAHHG_ERR_NOMEM = -6,     /* device or host allocation failed */
    GAHHG_ERR_STATE = -7,     /* call out of order (e.g. query before classify) */
    GAHHG_ERR_CAPACITY = -8   /* request exceeds a fixed maximum */
} gahhg_status;

typedef enum { GAHHG_SEMANTICS_EXACT = 0, GAHHG_SEMANTICS_REFERENCE = 1 } gahhg_semantics;

typedef enum {
    GAHHG_QUERY_AUTO = 0,          /* exact grids: FP32 filter; reference grids: FP64 */
    GAHHG_QUERY_FP32_FILTER = 1,   /* exact labels: FP32 certified filter -> FP64 -> expansion */
    GAHHG_QUERY_FP64_FILTER = 2,   /* exact labels: FP64 certified filter -> expansion */
    GAHHG_QUERY_REFERENCE_FP64 = 3 /* reference semantics: hierarchy descent in FP64 */
} gahhg_precision;

typedef struct gahhg_polygon gahhg_polygon;
typedef struct gahhg_points gahhg_points;
typedef struct gahhg_grid gahhg_grid;

typedef struct {
    int max_depth;      /* GPISPParam::maxDepth (source/GPISPParam.h:67), default 15 */
    int auto_depth;     /* GPISPParam::autoDepth (:68), default 1 */
    int semantics;      /* gahhg_semantics; GAHHG_SEMANTICS_EXACT builds both indexes */
    int lattice_top;    /* exact index: target number of top-level cells (0 = automatic, 8 per edge) */
    int lattice_leaf;   /* exact index: max edges per leaf before refining (0 = automatic) */
    int device;         /* CUDA device ordinal */
    int verbose;        /* print the reference's progress lines */
} gahhg_build_opts;

typedef struct {
    int depth;                 /* Depth of GAHHG (gnum) */
    int pv_num;                /* Number of polygon vertice */
    int vnum, bnum, cnum, rnum;
    int cpu_space;             /* sizeof(GAHHG)+28*gnum+sizeof(GPISPParam)+sizeof(GPISPStat) on x64 */
    int gpu_min_space;         /* 24 V + 48 B + 28 C + 4 R bytes */
    float gamma;
    double create_s;           /* createAHHGTime: level loop + edge dispatch */
    double classify_s;         /* classifyAHHGTime */
    double pre_s;              /* preTime = create + classify */
    double lattice_s;          /* exact index build (0 for reference semantics) */
    long long lattice_bytes;   /* device bytes of the exact index */
    double query_s;            /* PISPTime of the last gahhg_query* call */
    long long query_points;
    long long in_count;        /* labels == 2 in the last query */
    long long esc_fp64;        /* exact query: points the FP32 tier deferred to FP64 */
    long long esc_exact;       /* exact query: points the FP64 tier deferred to exact arithmetic */
    long long boundary_points; /* exact query: points that ran crossing tests */
    long long walk_limit_hits; /* edge walks stopped on a repeated state or at the step limit (the reference
                                  would not terminate) */
    long long scan_fallbacks;  /* build scans whose bounded look-back ran out and summed the late tile's
                                  inputs instead (exact either way; 0 in normal operation) */
} gahhg_stats;

/* Defaults as in GPISPParam::GPISPParam (source/GPISPParam.h:64-77). */
void gahhg_build_opts_init(gahhg_build_opts* o);

/* ---- loaders ------------------------------------------------------------ */

/* GPISPPolygon::loadPolyFromTXT (source/GPISPPolygon.cu:32-278): same
 * validation, the same messages on stdout, rings re-oriented so the outer
 * ring is counter-clockwise and holes clockwise (:209-264). */
gahhg_status gahhg_polygon_load(const char* path, gahhg_polygon** out);
/* In-memory variant: lonlat = 2 doubles per vertex, rings given without the
 * closing vertex, ring r spans vertices [ring_offsets[r], ring_offsets[r+1]),
 * ring 0 is the outer ring.  Same orientation rule as the file loader. */
gahhg_status gahhg_polygon_from_rings(const double* lonlat, const int64_t* ring_offsets, int nrings,
                                      gahhg_polygon** out);
int gahhg_polygon_num_edges(const gahhg_polygon* p);
/* Canonical vertex XYZ (3 doubles each) and edge list (2 ints each). */
gahhg_status gahhg_polygon_export(const gahhg_polygon* p, double* xyz, int* pe);
void gahhg_polygon_free(gahhg_polygon* p);

/* GPISPTP::loadTPFromCSV (source/GPISPTP.cu:13-79): "lon,lat" per line.
 * The file is parsed by all host threads; values and the first rejected line
 * are those of the reference's serial reading. */
gahhg_status gahhg_points_load(const char* path, gahhg_points** out);
/* The same with a binary sidecar `<path>.f64` (no counterpart in the
 * reference): GAHHG_POINTS_USE_SIDECAR reads the sidecar instead of the CSV
 * when it exists and matches the CSV's size and modification time;
 * GAHHG_POINTS_WRITE_SIDECAR writes it after parsing the CSV. */
#define GAHHG_POINTS_USE_SIDECAR 1
#define GAHHG_POINTS_WRITE_SIDECAR 2
gahhg_status gahhg_points_load_ex(const char* path, int flags, gahhg_points** out);
size_t gahhg_points_count(const gahhg_points* p);
const double* gahhg_points_lonlat(const gahhg_points* p);
void gahhg_points_free(gahhg_points* p);

/* ---- build / classify --------------------------------------------------- */

/* GPISP::createAHHGInit + createAHHG (source/GPISPAHHG.cu:1947-2015): the
 * level-synchronous refinement on the GPU plus the bottom-level edge lists.
 * For GAHHG_SEMANTICS_EXACT the build makes the exact-label lattice, which
 * exact queries use alone; the hexagon hierarchy is then built (and
 * classified) the first time gahhg_report_append, gahhg_grid_export,
 * gahhg_grid_depth or a GAHHG_QUERY_REFERENCE_FP64 query needs it, and until
 * then its fields of gahhg_stats are 0.  The polygon must outlive the grid. */
gahhg_status gahhg_build(const gahhg_polygon* poly, const gahhg_build_opts* opts, gahhg_grid** out);
/* GPISP::classifyAHHG (source/GPISPAHHG.cu:2018-2059). */
gahhg_status gahhg_classify(gahhg_grid* g);
void gahhg_grid_free(gahhg_grid* g);

/* ---- query -------------------------------------------------------------- */

/* GPISP::test / kernel_PISP (source/GPISPAHHG.cu:2062-2085, 1422-1504).
 * Device pointers: lonlat (2 doubles per point; 16-byte aligned for the
 * exact precisions, which read it in 16-byte units, else GAHHG_ERR_ARG),
 * labels (1 byte per point).
 * Asynchronous on `stream`; statistics are updated when `sync` is non-zero. */
gahhg_status gahhg_query_device(gahhg_grid* g, const double* d_lonlat, size_t n, uint8_t* d_labels,
                                int precision, void* stream, int sync);
/* Host pointers: copies lon/lat in, labels out, timing the kernel alone as
 * PISPTime does.  Synchronous. */
gahhg_status gahhg_query(gahhg_grid* g, const double* lonlat, size_t n, uint8_t* labels, int precision);

/* Same labels as gahhg_query_device, without allocating anything.  No
 * counterpart in the reference.
 *
 * For callers that cannot allocate device memory at query time: an
 * application that hands the whole device to its own allocator, a serving
 * loop that reserves all memory up front so a request can never fail on an
 * allocation, or code that must not hit the implicit synchronisation of
 * cudaMalloc/cudaFree.  gahhg_query_device takes its pass-2 scratch from a
 * stream-ordered pool; this variant uses a fixed 8 MB array in device memory
 * that the library reserves on every GPU that loads it, for as long as the
 * process lives.  Inputs and outputs are still the caller's device buffers.
 *
 * Limits: at most gahhg_query_noalloc_max_points() points per call (2,097,152;
 * more returns GAHHG_ERR_CAPACITY); exact grids only (GAHHG_QUERY_AUTO,
 * _FP32_FILTER or _FP64_FILTER); no statistics are collected.  Every call
 * asks the runtime for the array's device address (nothing is cached, so the
 * address stays right after a cudaDeviceReset); the first call on a device
 * also loads the library's kernels there, so make that first call before any
 * stream capture.  All calls share the one array and it keeps the
 * last call's contents: calls whose work overlaps on the GPU (two streams,
 * two host threads) race, so order them on one stream or serialise them. */
gahhg_status gahhg_query_device_noalloc(gahhg_grid* g, const double* d_lonlat, size_t n, uint8_t* d_labels,
                                        int precision, void* stream);
long long gahhg_query_noalloc_max_points(void);

/* ---- batches: many polygons (no counterpart in the reference) ----------- */

typedef struct gahhg_batch gahhg_batch;

typedef struct {
    int polygons;
    int workers;               /* host threads that built the groups of lattices */
    long long edges;
    long long lattice_bytes;   /* device bytes of all exact indexes */
    double build_s;            /* wall time of gahhg_batch_build */
    double query_s;            /* device time of the last synchronous batch query */
    long long query_points;
    long long boundary_points;
    long long esc_fp64;
    long long esc_exact;
    long long in_count;
} gahhg_batch_stats;

/* Builds the exact index of every polygon (exact semantics only; the hexagon
 * hierarchy is not built).  Consecutive polygons of up to 2^20 edges in all
 * are built together, each step once for the whole group; groups are built
 * concurrently on `workers` host threads (0 = up to 4), each with its own
 * stream.  The device memory pool keeps up to a quarter of the device's
 * memory cached from then on.  top_cells / leaf_edges, when not
 * NULL, set each polygon's lattice_top / lattice_leaf (e.g. from the
 * autotuner); 0 entries mean automatic.  The polygons must outlive the batch. */
gahhg_status gahhg_batch_build(const gahhg_polygon* const* polys, int count, const gahhg_build_opts* opts,
                               const int* top_cells, const int* leaf_edges, int workers, gahhg_batch** out);
int gahhg_batch_size(const gahhg_batch* b);
/* Points per work chunk of the persistent query launch (default 4096). */
gahhg_status gahhg_batch_set_chunk(gahhg_batch* b, int chunk_points);
/* Launch shapes of the query's first pass (the descent to a leaf): shape
 * `shape` runs `points_per_thread` points per thread in lockstep at
 * `blocks_per_sm` resident blocks of 256 threads per SM.  Shapes are numbered
 * from 0 (the default) until gahhg_batch_shape_info answers GAHHG_ERR_ARG.
 * Labels do not depend on the shape; the fastest depends on the batch's mix
 * of polygons and points (the autotuner measures them). */
gahhg_status gahhg_batch_shape_info(int shape, int* points_per_thread, int* blocks_per_sm);
gahhg_status gahhg_batch_set_shape(gahhg_batch* b, int shape);
/* Labels for all polygons at once.  d_lonlat holds the points polygon after
 * polygon: polygon p owns points [offsets[p], offsets[p+1]) (host array of
 * count+1 entries, offsets[0] = 0, fewer than 2^32 points in all).  Exact
 * labels (GAHHG_QUERY_AUTO, _FP32_FILTER, _FP64_FILTER).  Scratch comes from
 * the library's stream-ordered pool; with sync != 0 the call waits and
 * records statistics. */
gahhg_status gahhg_batch_query_device(gahhg_batch* b, const double* d_lonlat, const int64_t* offsets,
                                      uint8_t* d_labels, int precision, void* stream, int sync);
/* The same query as a CUDA graph: the first call with a given set of
 * pointers, offsets and precision captures the launch sequence (with its own
 * persistent scratch); later calls with the same arguments only launch the
 * graph on `stream`.  Replays of one batch's graph must not overlap. */
gahhg_status gahhg_batch_query_graph(gahhg_batch* b, const double* d_lonlat, const int64_t* offsets,
                                     uint8_t* d_labels, int precision, void* stream);
gahhg_status gahhg_batch_stats_get(const gahhg_batch* b, gahhg_batch_stats* s);
void gahhg_batch_free(gahhg_batch* b);

/* ---- serving: a request loop over resident indexes (no counterpart in the
 * reference, which answers one query file for one polygon per process) --- */

typedef struct gahhg_server gahhg_server;

typedef struct gahhg_server_opts {
    int device;
    int slots;              /* query batches in flight, each with its own stream and buffers (4) */
    long long slot_points;  /* points per batch; larger requests are split (4,194,304) */
    int max_pieces;         /* requests (or request pieces) per batch (4096) */
    int chunk_points;       /* work grain of the persistent query launch (4096) */
    int build_workers;      /* host threads building indexes, each with a low-priority stream (4) */
    int max_polygons;       /* polygon ids, resident or not (65536) */
    long long hbm_budget;   /* bytes of resident indexes; 0 = half the free device memory at creation */
    int evict_lru;          /* admit a build by evicting the least recently queried unpinned polygons */
    int precision;          /* GAHHG_QUERY_FP32_FILTER (default) or _FP64_FILTER; labels are exact either way */
    int direct_min_points;  /* requests in page-locked memory of at least this many points are copied
                               without staging (65536) */
} gahhg_server_opts;

/* Submission flags. */
#define GAHHG_SERVE_PINNED 1    /* build: never evicted to admit another build */
#define GAHHG_SERVE_DETACHED 2  /* no ticket is kept: the request cannot be waited on (drain instead) */

/* Polygon states (gahhg_server_polygon_state). */
#define GAHHG_POLY_FREE 0
#define GAHHG_POLY_QUEUED 1     /* waiting for HBM admission */
#define GAHHG_POLY_BUILDING 2
#define GAHHG_POLY_READY 3
#define GAHHG_POLY_FAILED 4
#define GAHHG_POLY_EVICTING 5   /* evicted; freed when its last query completes */

typedef struct gahhg_server_stats {
    long long queries_done;
    long long query_points;     /* points of completed queries */
    long long builds_done;
    long long builds_failed;    /* build errors and refused admissions */
    long long evictions;
    long long batches;          /* query batches launched */
    long long pieces;           /* request pieces in those batches */
    int resident_polygons;
    int pending_queries;
    int pending_builds;
    int inflight_batches;
    long long resident_bytes;   /* device bytes of resident indexes and polygons */
    long long hbm_budget;
    double window_s;            /* since creation or the last stats reset */
    double points_per_s;        /* query_points / window_s */
    double p50_ms, p90_ms, p99_ms, max_ms;  /* query latency, submission to labels in host memory */
    double build_p50_ms, build_p99_ms;      /* build latency, submission to ready */
    double mean_batch_points;
    double mean_batch_pieces;
    long long boundary_points;  /* points answered by the crossing test */
    long long esc_fp64;         /* crossing tests the FP32 filter could not decide */
    long long esc_exact;        /* ... nor the FP64 filter */
    long long in_count;
} gahhg_server_stats;

void gahhg_server_opts_init(gahhg_server_opts* o);
gahhg_status gahhg_server_create(const gahhg_server_opts* o, gahhg_server** out);
/* Queues the exact-index build of a copy of `poly` (the handle may be freed
 * after the call).  *id is the polygon's id at once: queries to it are held
 * until it is ready.  A build is admitted when its estimated footprint fits
 * in the budget; one that cannot fit even after eviction fails with
 * GAHHG_ERR_CAPACITY on its ticket.  Ids are reused after eviction. */
gahhg_status gahhg_server_submit_build(gahhg_server* s, const gahhg_polygon* poly, int top_cells, int leaf_edges,
                                       int flags, int* id, int64_t* ticket);
/* Queues labels for n points (host lon/lat pairs) of polygon `id`, written
 * to labels[0..n) before the request completes.  Both buffers must stay
 * valid until then.  Requests are batched with whatever else is pending
 * when a slot frees, so work of concurrent requests overlaps on the device;
 * a request's labels do not depend on what it was batched with. */
gahhg_status gahhg_server_submit_query(gahhg_server* s, int id, const double* lonlat, int64_t n, uint8_t* labels,
                                       int flags, int64_t* ticket);
/* Waits for a ticket: returns the request's own status (and forgets the
 * ticket), or GAHHG_ERR_STATE if it is still pending after timeout_s. */
gahhg_status gahhg_server_wait(gahhg_server* s, int64_t ticket, double timeout_s);
/* Waits until no request is pending or in flight (GAHHG_ERR_STATE on timeout). */
gahhg_status gahhg_server_drain(gahhg_server* s, double timeout_s);
/* Frees polygon `id` once its submitted queries complete; later queries to
 * it fail.  Also releases the id of a failed build. */
gahhg_status gahhg_server_evict(gahhg_server* s, int id);
gahhg_status gahhg_server_polygon_state(gahhg_server* s, int id, int* state, long long* bytes);
gahhg_status gahhg_server_stats_get(gahhg_server* s, gahhg_server_stats* out);
/* Clears latency samples and counters and restarts the window. */
gahhg_status gahhg_server_stats_reset(gahhg_server* s);
/* Copies up to `cap` latency samples (ms) of kind 0 = queries, 1 = builds;
 * returns how many there are. */
long long gahhg_server_latencies(gahhg_server* s, int kind, double* out, long long cap);
/* Per-batch trace (kind 0 = query batches): up to `cap` records of 6 doubles
 * each - formed (s since the window start), host enqueue ms, device ms,
 * completion ms after forming, points, pieces.  Returns the record count. */
long long gahhg_server_trace(gahhg_server* s, double* out, long long cap);
/* Host-side stalls of 2 ms or more since the last stats reset: up to `cap`
 * records of 3 doubles - start (s since the window start), kind, ms.  Kinds:
 * 1 waiting for the server lock at submission, 2 the page-locked memory
 * query at submission, 3 freeing an evicted polygon, 4 admission, 5 a build,
 * 6 a view upload, 7 enqueueing a batch, 8 copying a batch's labels out.
 * Returns the record count. */
long long gahhg_server_stalls(gahhg_server* s, double* out, long long cap);
/* Drains (up to 60 s), stops the threads and frees everything. */
void gahhg_server_free(gahhg_server* s);

/* ---- statistics / report ------------------------------------------------ */

gahhg_status gahhg_stats_get(const gahhg_grid* g, gahhg_stats* s);
/* Level table: 7 ints per level (vstart vnum bstart bnum cstart cnum rnum). */
int gahhg_grid_depth(const gahhg_grid* g);
/* Grid arrays for inspection: levels, vertices (3 doubles), borders (48 B),
 * cells (28 B), bottom-level refs.  Any pointer may be NULL. */
gahhg_status gahhg_grid_export(const gahhg_grid* g, int* levels, double* v, void* b, void* c, int* refs);
/* GPISP::exportStat2TXT (source/GPISPAHHG.cu:2115-2161): appends the report
 * block to `path` (dest_stdout != 0 prints it instead). */
gahhg_status gahhg_report_append(const gahhg_grid* g, const char* polyfile, const char* tpfile,
                                 long long npoints, const char* path, int dest_stdout);
/* GPISPTP::exportResult2CSV (source/GPISPTP.cu:81-99). */
gahhg_status gahhg_result_write(const char* path, const uint8_t* labels, size_t n);

/* The level-0 grid (80 vertices, 240 borders, 42 cells). */
gahhg_status gahhg_grid0_export(double* v, void* b, void* c);

/* Blocks on `device` whose bulk copy (TMA) into shared memory did not
 * complete within the bounded wait, since the library was loaded: pass-1
 * (locate) blocks staging the coarse summary, and tier-1 blocks staging a
 * tile's leaf and edge records (pass-2 order 3).  Such a block loads the
 * data with plain loads instead, so labels are unaffected; 0 in normal
 * operation. */
gahhg_status gahhg_staging_fallbacks(int device, unsigned long long* count);

/* Process-wide tuning and test knobs.  No counterpart in the reference.
 * GAHHG_KNOB_GROUPED_PASS2: the order in which the crossing tests take the
 * points that pass 1 of a single-polygon exact query could not label, when
 * there are at least 2^18 of them: 0 (default) input order; 1 windows of
 * consecutive leaves (about 24 MB of index each; only when the index spans
 * several windows); 2 leaf order (a counting sort by leaf); 3 leaf order, with
 * the first (FP32) tier reading each tile's leaf and edge records from shared
 * memory, where one bulk copy (TMA) per tile staged them.  Labels are the
 * same in every order.
 * Values take effect for work enqueued after the call. */
typedef enum {
    GAHHG_KNOB_GROUPED_PASS2 = 1,
    /* Bounded waits and loops, lowered by tests to make them run out (never
     * needed otherwise; 0 or more, defaults in brackets):
     * WALK_STEP_LIMIT     cells an edge walk of the hierarchy visits before it
     *                     stops and counts a walk_limit_hit [65,536];
     * SCAN_SPIN_LIMIT     polls a build scan's look-back waits for an earlier
     *                     tile before summing that tile's inputs itself
     *                     (counted in scan_fallbacks) [4,194,304];
     * STAGING_POLL_LIMIT  polls a pass-1 block waits for the bulk copy of the
     *                     coarse summary, and a staging tier-1 block for a
     *                     tile's records, before reading global memory instead
     *                     (counted by gahhg_staging_fallbacks) [1,048,576]. */
    GAHHG_KNOB_WALK_STEP_LIMIT = 2,
    GAHHG_KNOB_SCAN_SPIN_LIMIT = 3,
    GAHHG_KNOB_STAGING_POLL_LIMIT = 4
} gahhg_knob;
gahhg_status gahhg_set_knob(int knob, long long value);
long long gahhg_get_knob(int knob);

const char* gahhg_last_error(void);
int gahhg_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* GAHHG_H */
