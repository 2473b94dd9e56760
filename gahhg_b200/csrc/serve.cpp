// serve.cpp - a request loop over resident exact indexes (include/gahhg.h,
// gahhg_server_*).
//
// No counterpart in the reference: its program answers one query file for
// one polygon per process (source/GPISP.cu:15-70).  Here indexes stay on the
// device and requests arrive continuously from any number of host threads.
//
// Queries.  A dispatcher thread forms a batch whenever a slot is free: it
// takes pending requests in arrival order (splitting one that does not fit)
// up to the slot's point capacity, so requests that arrived while earlier
// batches were on the device ride the next free slot (continuous batching).
// Each slot owns a high-priority stream, a page-locked staging area and
// device buffers laid out as
//
//     [labels (LCAP B)][header 64 B][chunk table][points (16 B each)]
//
// so a batch is one host-to-device copy (header zeros, chunk table, staged
// points), the two query kernels (the persistent chunked locate pass and the
// leaf pass, which find each point's polygon through the chunk table), and
// one device-to-host copy of [labels of this batch][header with counters]:
// the labels of a batch of n points occupy the last n bytes before the
// header.  Requests in page-locked memory skip the staging copy.  Slots run
// concurrently, so one batch's copies overlap another's kernels.  A
// completion thread polls the slots' events, copies labels out and records
// each request's latency (submission to labels in host memory).
//
// Builds.  Build workers (low-priority streams) take queued builds in order
// once their estimated footprint fits in the HBM budget, evicting least
// recently queried unpinned polygons first when asked to.  The estimate
// (bytes per edge, learnt from finished builds, with a margin) is replaced by
// the measured footprint when the build finishes.  Queries to a polygon that
// is still building are held and released when it is ready.
//
// A polygon's reference count covers its submitted but unfinished queries,
// so an evicted polygon is freed only after the last of them completes.
#include <algorithm>
#include <array>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "gahhg_internal.h"

using namespace gahhg;

namespace {

constexpr size_t HDR_BYTES = 64;  // [u32 queue count, next chunk, tier counters x3][u64 stats x4 at +32]
constexpr size_t CHUNK_BYTES = 16;
constexpr int MAX_SUMMARY_WORDS = 4096;  // the batch kernel stages at most 16 KB of summary
constexpr size_t MAX_TRACE = 1 << 20;
constexpr double STALL_MS = 2.0;
// stall kinds (gahhg_server_stalls)
enum { STALL_SUBMIT_LOCK = 1, STALL_POINTER_QUERY = 2, STALL_FREE = 3, STALL_ADMIT = 4, STALL_BUILD = 5,
       STALL_VIEW_UPLOAD = 6, STALL_LAUNCH = 7, STALL_COPY_OUT = 8 };

struct Req {
    int64_t ticket = 0;
    bool build = false;
    bool detached = false;
    bool direct = false;  // page-locked points: no staging copy
    int poly = -1;
    const double* lonlat = nullptr;
    uint8_t* labels = nullptr;
    int64_t n = 0;
    int64_t next = 0;  // first point not yet in a batch
    int inflight = 0;  // pieces in batches not yet completed
    double t_submit = 0.0;
    gahhg_status status = GAHHG_OK;
    std::string msg;  // error text of a failed request
    bool done = false;
};

struct Piece {
    Req* r;
    int64_t a, n;  // points [a, a + n) of the request
    int64_t dev;   // first point in the slot's point array
};

struct SrvPoly {
    int state = GAHHG_POLY_FREE;
    std::unique_ptr<Polygon> poly;
    Grid* grid = nullptr;
    int top = 0, leaf = 0;
    bool pinned = false;
    int refs = 0;         // submitted queries not yet completed
    long long est = 0;    // admission estimate (while queued or building)
    long long bytes = 0;  // measured device bytes (when ready)
    double last_use = 0.0;
    int swords = 0;
    Req* build_req = nullptr;
    std::vector<Req*> held;  // queries waiting for the build
};

struct Slot {
    cudaStream_t s = nullptr;
    cudaEvent_t ev0 = nullptr, ev = nullptr;
    uint8_t* h = nullptr;  // page-locked, same layout as d
    uint8_t* d = nullptr;
    uint32_t* d_queue = nullptr;
    std::vector<Piece> pieces;
    std::vector<int> seg_view, swords;
    std::vector<long long> seg_off;
    int64_t points = 0;
    double t_form = 0.0, t_enq = 0.0;
    bool busy = false;
};

double percentile(std::vector<double> v, double q)
{
    if (v.empty()) return 0.0;
    const size_t k = std::min(v.size() - 1, (size_t)(q * (double)(v.size() - 1) + 0.5));
    std::nth_element(v.begin(), v.begin() + k, v.end());
    return v[k];
}

}  // namespace

struct gahhg_server {
    gahhg_server_opts o{};
    gahhg_build_opts base{};
    size_t lcap = 0, in_bytes = 0, cap_chunks = 0;

    std::mutex mu;
    std::condition_variable cv_dispatch, cv_complete, cv_build, cv_wait;
    bool stop = false;
    bool broken = false;
    std::string broken_msg;

    std::vector<SrvPoly> polys;
    std::vector<int> free_ids;
    int next_id = 0;
    uint8_t* d_views = nullptr;
    size_t view_bytes = 0;

    std::deque<Req*> pending;     // dispatchable queries
    std::deque<int> build_queue;  // polygon ids awaiting admission
    std::unordered_map<int64_t, Req*> tickets;
    int64_t next_ticket = 1;
    long long outstanding = 0;  // requests submitted and not completed

    std::vector<Slot> slots;
    std::vector<Slot*> inflight;
    WorkerPool workers;
    int builds_running = 0;
    long long committed = 0;         // resident bytes + estimates of running builds
    double bytes_per_edge = 1024.0;  // learnt estimate
    long long resident_bytes = 0;
    int resident = 0;

    std::thread dispatcher, completer;
    std::vector<std::thread> builders;

    // statistics since the last reset
    double t0 = 0.0;
    std::vector<double> lat_q, lat_b;
    std::vector<std::array<double, 6>> trace;
    // Objects released under the server lock are freed after it is dropped:
    // freeing makes CUDA calls, and a driver call can wait behind another
    // thread's (a pool growing, say) for hundreds of milliseconds; nothing
    // that submissions wait for may hold the lock meanwhile.
    // A reaper thread frees them, so no thread on the query path waits either.
    std::mutex grave_mu;
    std::condition_variable cv_grave;
    bool grave_stop = false;
    std::vector<Grid*> grave_grids;
    std::vector<std::unique_ptr<Polygon>> grave_polys;
    std::thread reaper;
    void bury_locked(SrvPoly& P)
    {
        {
            std::lock_guard<std::mutex> lk(grave_mu);
            if (P.grid) grave_grids.push_back(P.grid);
            if (P.poly) grave_polys.push_back(std::move(P.poly));
        }
        P.grid = nullptr;
        P.poly.reset();
        cv_grave.notify_one();
    }
    void reap_loop()
    {
        cudaSetDevice(o.device);
        std::unique_lock<std::mutex> lk(grave_mu);
        for (;;) {
            cv_grave.wait(lk, [&] { return grave_stop || !grave_grids.empty() || !grave_polys.empty(); });
            std::vector<Grid*> g;
            std::vector<std::unique_ptr<Polygon>> p;
            g.swap(grave_grids);
            p.swap(grave_polys);
            const bool last = grave_stop;
            lk.unlock();
            if (!g.empty() || !p.empty()) {
                const double tf = now_seconds();
                for (Grid* x : g) delete x;
                p.clear();
                note_stall(STALL_FREE, tf, now_seconds());
            }
            lk.lock();
            if (last && grave_grids.empty() && grave_polys.empty()) break;
        }
    }

    // host-side stalls above STALL_MS: (seconds since the window start, kind, ms)
    std::mutex stall_mu;
    std::vector<std::array<double, 3>> stalls;
    void note_stall(int kind, double t_begin, double t_end)
    {
        const double ms = (t_end - t_begin) * 1e3;
        if (ms < STALL_MS) return;
        std::lock_guard<std::mutex> lk(stall_mu);
        if (stalls.size() < MAX_TRACE) stalls.push_back({t_begin - t0, (double)kind, ms});
    }
    long long queries_done = 0, query_points = 0, builds_done = 0, builds_failed = 0, evictions = 0;
    long long batches = 0, pieces = 0, batch_points = 0;
    long long st_boundary = 0, st_fp64 = 0, st_exact = 0, st_in = 0;

    // ------------------------------------------------------------------
    void complete_locked(Req* r, gahhg_status st)
    {
        r->done = true;
        if (r->status == GAHHG_OK) r->status = st;
        if (r->status != GAHHG_OK && r->msg.empty()) r->msg = last_error();
        const double ms = (now_seconds() - r->t_submit) * 1e3;
        if (r->build) {
            lat_b.push_back(ms);
        } else {
            lat_q.push_back(ms);
            queries_done++;
            if (r->status == GAHHG_OK) query_points += r->n;
            if (r->poly >= 0) unref_locked(r->poly);
        }
        outstanding--;
        if (r->detached) delete r;
        cv_wait.notify_all();
    }

    void unref_locked(int id)
    {
        SrvPoly& P = polys[id];
        if (--P.refs == 0 && P.state == GAHHG_POLY_EVICTING) free_poly_locked(id);
    }

    void free_poly_locked(int id)
    {
        SrvPoly& P = polys[id];
        bury_locked(P);
        committed -= P.bytes;
        resident_bytes -= P.bytes;
        resident--;
        P.bytes = 0;
        P.state = GAHHG_POLY_FREE;
        evictions++;
        free_ids.push_back(id);
        cv_build.notify_all();
    }

    long long estimate(long long edges) const
    {
        // lattice + polygon copy (24 B vertex + 8 B edge), 256 KB floor, 1.5x margin
        return std::max<long long>(256 << 10, (long long)(1.5 * bytes_per_edge * (double)edges)) + edges * 32;
    }

    // ------------------------------------------------------------- queries --
    void dispatch_loop()
    {
        cudaSetDevice(o.device);
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            cv_dispatch.wait(lk, [&] {
                if (stop) return true;
                if (pending.empty()) return false;
                if (broken) return true;
                for (Slot& s : slots)
                    if (!s.busy) return true;
                return false;
            });
            if (stop) break;
            if (broken) {
                while (!pending.empty()) {
                    Req* r = pending.front();
                    pending.pop_front();
                    r->next = r->n;
                    if (r->inflight == 0)
                        complete_locked(r, GAHHG_ERR_CUDA);
                    else
                        r->status = GAHHG_ERR_CUDA;
                }
                continue;
            }
            Slot* sl = nullptr;
            for (Slot& s : slots)
                if (!s.busy) {
                    sl = &s;
                    break;
                }
            sl->busy = true;
            sl->pieces.clear();
            int64_t pts = 0;
            const double now = now_seconds();
            sl->t_form = now;
            while (!pending.empty() && (int)sl->pieces.size() < o.max_pieces && pts < o.slot_points) {
                Req* r = pending.front();
                const int64_t take = std::min<int64_t>(r->n - r->next, o.slot_points - pts);
                sl->pieces.push_back(Piece{r, r->next, take, 0});
                r->next += take;
                r->inflight++;
                pts += take;
                polys[r->poly].last_use = now;
                if (r->next == r->n) pending.pop_front();
            }
            // staged pieces first, then the ones copied straight from
            // page-locked memory; views and summary sizes are read under the
            // lock (the polygons stay resident while these requests hold
            // references)
            std::stable_partition(sl->pieces.begin(), sl->pieces.end(), [](const Piece& p) { return !p.r->direct; });
            sl->seg_view.clear();
            sl->swords.clear();
            for (const Piece& p : sl->pieces) {
                sl->seg_view.push_back(p.r->poly);
                sl->swords.push_back(polys[p.r->poly].swords);
            }
            sl->points = pts;
            lk.unlock();
            const double tl = now_seconds();
            const gahhg_status st = launch(sl);
            sl->t_enq = now_seconds();
            note_stall(STALL_LAUNCH, tl, sl->t_enq);
            lk.lock();
            batches++;
            pieces += (long long)sl->pieces.size();
            batch_points += pts;
            if (st != GAHHG_OK) {
                fail_slot_locked(sl, st);
                continue;
            }
            inflight.push_back(sl);
            cv_complete.notify_one();
        }
    }

    // Stages and enqueues one batch (no lock held; the slot is ours).
    gahhg_status launch(Slot* sl)
    {
        const int nseg = (int)sl->pieces.size();
        sl->seg_off.assign(nseg + 1, 0);
        int64_t staged = 0;
        for (int i = 0; i < nseg; i++) {
            Piece& p = sl->pieces[i];
            p.dev = sl->seg_off[i];
            sl->seg_off[i + 1] = sl->seg_off[i] + p.n;
            if (!p.r->direct) staged += p.n;
        }
        int nchunks = 0;
        batch_write_chunks(sl->seg_off.data(), nseg, o.chunk_points, sl->swords.data(), sl->seg_view.data(), nullptr,
                           &nchunks);
        if ((size_t)nchunks > cap_chunks) {
            set_error("server batch needs %d chunks (capacity %zu)", nchunks, cap_chunks);
            return GAHHG_ERR_CAPACITY;
        }
        uint8_t* hin = sl->h + lcap;
        memset(hin, 0, HDR_BYTES);
        batch_write_chunks(sl->seg_off.data(), nseg, o.chunk_points, sl->swords.data(), sl->seg_view.data(),
                           hin + HDR_BYTES, &nchunks);
        const size_t pts_off = HDR_BYTES + (size_t)nchunks * CHUNK_BYTES;
        double* hp = (double*)(hin + pts_off);
        for (const Piece& p : sl->pieces)
            if (!p.r->direct) memcpy(hp + 2 * p.dev, p.r->lonlat + 2 * p.a, (size_t)p.n * 16);
        uint8_t* din = sl->d + lcap;
        GAHHG_CUDA_TRY(cudaEventRecord(sl->ev0, sl->s));
        GAHHG_CUDA_TRY(cudaMemcpyAsync(din, hin, pts_off + (size_t)staged * 16, cudaMemcpyHostToDevice, sl->s));
        for (const Piece& p : sl->pieces)
            if (p.r->direct)
                GAHHG_CUDA_TRY(cudaMemcpyAsync(din + pts_off + (size_t)p.dev * 16, p.r->lonlat + 2 * p.a,
                                               (size_t)p.n * 16, cudaMemcpyHostToDevice, sl->s));
        // labels end where the header starts, so one copy brings both back
        uint8_t* d_labels = sl->d + lcap - (size_t)sl->points;
        GAHHG_TRY(batch_query_launch(d_views, din + HDR_BYTES, nchunks, (const double*)(din + pts_off), d_labels,
                                     o.precision, sl->d_queue, o.slot_points, (unsigned int*)din,
                                     (uint64_t*)(din + 32), sl->s,
                                     o.device, false));
        GAHHG_CUDA_TRY(cudaMemcpyAsync(sl->h + lcap - (size_t)sl->points, d_labels, (size_t)sl->points + HDR_BYTES,
                                       cudaMemcpyDeviceToHost, sl->s));
        GAHHG_CUDA_TRY(cudaEventRecord(sl->ev, sl->s));
        return GAHHG_OK;
    }

    void fail_slot_locked(Slot* sl, gahhg_status st)
    {
        for (const Piece& p : sl->pieces) {
            Req* r = p.r;
            r->status = st;
            if (--r->inflight == 0 && r->next == r->n) complete_locked(r, st);
        }
        sl->pieces.clear();
        sl->busy = false;
        cv_dispatch.notify_one();
    }

    void complete_loop()
    {
        cudaSetDevice(o.device);
        std::unique_lock<std::mutex> lk(mu);
        std::vector<Slot*> snap;
        for (;;) {
            cv_complete.wait(lk, [&] { return stop || !inflight.empty(); });
            if (inflight.empty()) {
                if (stop) break;
                continue;
            }
            snap = inflight;
            lk.unlock();
            Slot* done = nullptr;
            cudaError_t err = cudaSuccess;
            for (Slot* s : snap) {
                const cudaError_t e = cudaEventQuery(s->ev);
                if (e != cudaErrorNotReady) {
                    done = s;
                    err = e;
                    break;
                }
            }
            if (!done) {
                std::this_thread::yield();
                lk.lock();
                continue;
            }
            float dev_ms = 0.f;
            if (err == cudaSuccess) {
                const double tc = now_seconds();
                const uint8_t* lab = done->h + lcap - (size_t)done->points;
                for (const Piece& p : done->pieces) memcpy(p.r->labels + p.a, lab + p.dev, (size_t)p.n);
                cudaEventElapsedTime(&dev_ms, done->ev0, done->ev);
                note_stall(STALL_COPY_OUT, tc, now_seconds());
            }
            const double t_done = now_seconds();
            lk.lock();
            inflight.erase(std::find(inflight.begin(), inflight.end(), done));
            if (err != cudaSuccess) {
                broken = true;
                broken_msg = cudaGetErrorString(err);
                set_error("server batch failed: %s", broken_msg.c_str());
                fail_slot_locked(done, GAHHG_ERR_CUDA);
                cv_dispatch.notify_all();
                continue;
            }
            const uint64_t* c = (const uint64_t*)(done->h + lcap + 32);
            st_fp64 += (long long)c[0];
            st_exact += (long long)c[1];
            st_boundary += (long long)c[2];
            st_in += (long long)c[3];
            if (trace.size() < MAX_TRACE)
                trace.push_back({done->t_form - t0, (done->t_enq - done->t_form) * 1e3, (double)dev_ms,
                                 (t_done - done->t_form) * 1e3, (double)done->points, (double)done->pieces.size()});
            for (const Piece& p : done->pieces) {
                Req* r = p.r;
                if (--r->inflight == 0 && r->next == r->n) complete_locked(r, GAHHG_OK);
            }
            done->pieces.clear();
            done->busy = false;
            cv_dispatch.notify_one();
        }
    }

    // -------------------------------------------------------------- builds --
    // Next admitted build, or -1 (wait).  Refusals complete here.
    int admit_locked()
    {
        while (!build_queue.empty()) {
            const int id = build_queue.front();
            SrvPoly& P = polys[id];
            const long long need = P.est;
            if (committed + need <= o.hbm_budget) {
                build_queue.pop_front();
                committed += need;
                P.state = GAHHG_POLY_BUILDING;
                builds_running++;
                return id;
            }
            if (o.evict_lru) {
                // least recently queried, unpinned, unused polygons first
                std::vector<int> cand;
                for (int i = 0; i < next_id; i++) {
                    const SrvPoly& Q = polys[i];
                    if (Q.state == GAHHG_POLY_READY && !Q.pinned && Q.refs == 0) cand.push_back(i);
                }
                std::sort(cand.begin(), cand.end(),
                          [&](int a, int b) { return polys[a].last_use < polys[b].last_use; });
                for (int i : cand) {
                    if (committed + need <= o.hbm_budget) break;
                    free_poly_locked(i);
                }
                if (committed + need <= o.hbm_budget) continue;
            }
            // wait only while something under way can release memory
            bool can_free = builds_running > 0;
            for (int i = 0; i < next_id && !can_free; i++) {
                const SrvPoly& Q = polys[i];
                if (Q.state == GAHHG_POLY_EVICTING) can_free = true;
                if (o.evict_lru && Q.state == GAHHG_POLY_READY && !Q.pinned && Q.refs > 0) can_free = true;
            }
            if (need <= o.hbm_budget && can_free) return -1;
            build_queue.pop_front();
            set_error("build of %lld estimated bytes does not fit in the HBM budget (%lld of %lld committed)", need,
                      committed, o.hbm_budget);
            fail_build_locked(id, GAHHG_ERR_CAPACITY);
        }
        return -1;
    }

    void fail_build_locked(int id, gahhg_status st)
    {
        SrvPoly& P = polys[id];
        P.state = GAHHG_POLY_FAILED;
        builds_failed++;
        for (Req* r : P.held) {
            r->next = r->n;
            complete_locked(r, st);
        }
        P.held.clear();
        if (P.build_req) complete_locked(P.build_req, st);
        P.build_req = nullptr;
        bury_locked(P);
    }

    void build_loop(int w)
    {
        cudaSetDevice(o.device);
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            int id = -1;
            cv_build.wait(lk, [&] {
                if (stop) return true;
                const double ta = now_seconds();
                id = admit_locked();
                note_stall(STALL_ADMIT, ta, now_seconds());
                return id >= 0;
            });
            if (stop && id < 0) break;
            SrvPoly& P = polys[id];
            Polygon* poly = P.poly.get();
            const int top = P.top, leaf = P.leaf;
            lk.unlock();
            Grid* g = nullptr;
            const double tb = now_seconds();
            gahhg_status st =
                build_exact_grid(poly, o.device, workers.streams[w], &workers.scans[w], base, top, leaf, &g);
            note_stall(STALL_BUILD, tb, now_seconds());
            int sw = 0;
            long long bytes = 0;
            std::string msg;
            if (st == GAHHG_OK) {
                sw = (int)lattice_summary_words(g);
                if (sw > MAX_SUMMARY_WORDS) {
                    set_error("the index's coarse summary (%d words) exceeds the batch kernel's %d", sw,
                              MAX_SUMMARY_WORDS);
                    st = GAHHG_ERR_CAPACITY;
                }
            }
            if (st == GAHHG_OK) {
                std::vector<uint8_t> v(view_bytes);
                lattice_view_write(g, v.data());
                cudaStream_t ws = workers.streams[w];
                const double tv = now_seconds();
                if (cudaMemcpyAsync(d_views + (size_t)id * view_bytes, v.data(), view_bytes, cudaMemcpyHostToDevice,
                                    ws) != cudaSuccess ||
                    cudaStreamSynchronize(ws) != cudaSuccess) {
                    set_error("view upload: %s", cudaGetErrorString(cudaGetLastError()));
                    st = GAHHG_ERR_CUDA;
                }
                note_stall(STALL_VIEW_UPLOAD, tv, now_seconds());
                bytes = (long long)lattice_device_bytes(g->lattice) + (long long)poly->pv_num * 32;
            }
            if (st != GAHHG_OK) {
                msg = last_error();
                delete g;
                g = nullptr;
            }
            lk.lock();
            builds_running--;
            committed -= P.est;
            if (st != GAHHG_OK) {
                set_error("%s", msg.c_str());
                fail_build_locked(id, st);
            } else {
                P.grid = g;
                P.swords = sw;
                P.bytes = bytes;
                committed += bytes;
                resident_bytes += bytes;
                resident++;
                P.state = GAHHG_POLY_READY;
                builds_done++;
                if (poly->pv_num > 0) {
                    const double bpe = (double)(bytes - (long long)poly->pv_num * 32) / (double)poly->pv_num;
                    // never below the newest observation; decays slowly from larger ones
                    bytes_per_edge = std::max(bpe, 0.9 * bytes_per_edge + 0.1 * bpe);
                }
                for (Req* r : P.held) pending.push_back(r);
                if (!P.held.empty()) cv_dispatch.notify_one();
                P.held.clear();
                if (P.build_req) complete_locked(P.build_req, GAHHG_OK);
                P.build_req = nullptr;
            }
            cv_build.notify_all();
        }
    }

    // ---------------------------------------------------------- lifecycle --
    gahhg_status init()
    {
        GAHHG_CUDA_TRY(cudaSetDevice(o.device));
        gahhg_build_opts_init(&base);
        base.device = o.device;
        base.semantics = GAHHG_SEMANTICS_EXACT;
        view_bytes = lattice_view_bytes();
        polys.resize(o.max_polygons);
        GAHHG_CUDA_TRY(cudaMalloc(&d_views, view_bytes * (size_t)o.max_polygons));
        lcap = ((size_t)o.slot_points + 63) & ~(size_t)63;
        cap_chunks = batch_chunk_count_bound(o.slot_points, o.max_pieces, o.chunk_points);
        in_bytes = HDR_BYTES + cap_chunks * CHUNK_BYTES + (size_t)o.slot_points * 16;
        int lo = 0, hi = 0;
        cudaDeviceGetStreamPriorityRange(&lo, &hi);  // hi is the greatest priority (numerically lowest)
        slots.resize(o.slots);
        for (Slot& s : slots) {
            GAHHG_CUDA_TRY(cudaStreamCreateWithPriority(&s.s, cudaStreamNonBlocking, hi));
            GAHHG_CUDA_TRY(cudaEventCreate(&s.ev0));
            GAHHG_CUDA_TRY(cudaEventCreate(&s.ev));
            GAHHG_CUDA_TRY(cudaHostAlloc((void**)&s.h, lcap + in_bytes, cudaHostAllocDefault));
            GAHHG_CUDA_TRY(cudaMalloc((void**)&s.d, lcap + in_bytes));
            GAHHG_CUDA_TRY(cudaMalloc((void**)&s.d_queue, sizeof(uint32_t) * batch_queue_words(o.slot_points)));
        }
        GAHHG_TRY(workers.create(o.device, o.build_workers, lo));
        if (o.hbm_budget <= 0) {
            size_t fr = 0, tot = 0;
            GAHHG_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
            o.hbm_budget = (long long)(fr / 2);
        }
        // the budget stays mapped in the pool between builds: returning
        // freed memory to the driver and mapping it again on the next build
        // would churn page mappings while queries run
        GAHHG_TRY(pool_keep(o.device, (size_t)o.hbm_budget + (4ull << 30)));
        // map the budget into the pool once, up front: growing the pool
        // while serving maps physical memory, and every build thread's
        // allocations waited for it (half-second stalls of all builds)
        {
            size_t fr = 0, tot = 0;
            GAHHG_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
            const size_t want = std::min<size_t>((size_t)o.hbm_budget + ((size_t)4 << 30), (size_t)(0.9 * (double)fr));
            void* p = nullptr;
            cudaStream_t s0 = workers.streams[0];
            if (want > 0 && pool_alloc(&p, want, o.device, s0) == GAHHG_OK) {
                cudaFreeAsync(p, s0);
                cudaStreamSynchronize(s0);
            }
            cudaGetLastError();
        }
        t0 = now_seconds();
        dispatcher = std::thread([this] { dispatch_loop(); });
        completer = std::thread([this] { complete_loop(); });
        reaper = std::thread([this] { reap_loop(); });
        for (int w = 0; w < o.build_workers; w++) builders.emplace_back([this, w] { build_loop(w); });
        return GAHHG_OK;
    }

    gahhg_status drain(double timeout_s)
    {
        std::unique_lock<std::mutex> lk(mu);
        if (!cv_wait.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return outstanding == 0; })) {
            set_error("drain: %lld requests still pending", outstanding);
            return GAHHG_ERR_STATE;
        }
        return GAHHG_OK;
    }

    ~gahhg_server()
    {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv_dispatch.notify_all();
        cv_complete.notify_all();
        cv_build.notify_all();
        if (dispatcher.joinable()) dispatcher.join();
        for (auto& t : builders)
            if (t.joinable()) t.join();
        // batches already launched finish before their slots go away
        for (Slot& s : slots)
            if (s.s) cudaStreamSynchronize(s.s);
        {
            std::lock_guard<std::mutex> lk(mu);
            cv_complete.notify_all();
        }
        if (completer.joinable()) completer.join();
        cudaSetDevice(o.device);
        for (Slot& s : slots) {
            if (s.ev0) cudaEventDestroy(s.ev0);
            if (s.ev) cudaEventDestroy(s.ev);
            if (s.s) cudaStreamDestroy(s.s);
            if (s.h) cudaFreeHost(s.h);
            if (s.d) cudaFree(s.d);
            if (s.d_queue) cudaFree(s.d_queue);
        }
        {
            std::lock_guard<std::mutex> lk(grave_mu);
            grave_stop = true;
        }
        cv_grave.notify_all();
        if (reaper.joinable()) reaper.join();
        for (SrvPoly& P : polys) {
            delete P.grid;
            P.grid = nullptr;
            P.poly.reset();
            for (Req* r : P.held)
                if (r->detached) delete r;
            if (P.build_req && P.build_req->detached) delete P.build_req;
        }
        for (auto& kv : tickets) delete kv.second;
        for (Req* r : pending)
            if (r->detached) delete r;
        workers.destroy();
        if (d_views) cudaFree(d_views);
    }
};

extern "C" {

void gahhg_server_opts_init(gahhg_server_opts* o)
{
    if (!o) return;
    memset(o, 0, sizeof(*o));
    o->device = 0;
    o->slots = 4;
    o->slot_points = 1LL << 22;
    o->max_pieces = 4096;
    o->chunk_points = 4096;
    o->build_workers = 4;
    o->max_polygons = 65536;
    o->hbm_budget = 0;
    o->evict_lru = 0;
    o->precision = GAHHG_QUERY_FP32_FILTER;
    o->direct_min_points = 65536;
}

gahhg_status gahhg_server_create(const gahhg_server_opts* opts, gahhg_server** out)
{
    if (!out) return GAHHG_ERR_ARG;
    *out = nullptr;
    gahhg_server_opts o;
    if (opts)
        o = *opts;
    else
        gahhg_server_opts_init(&o);
    if (o.precision == GAHHG_QUERY_AUTO) o.precision = GAHHG_QUERY_FP32_FILTER;
    if (o.slots < 1 || o.slots > 64 || o.slot_points < 1024 || o.slot_points > (1LL << 31) || o.max_pieces < 1 ||
        o.chunk_points < 256 || o.build_workers < 1 || o.build_workers > 64 || o.max_polygons < 1 ||
        (o.precision != GAHHG_QUERY_FP32_FILTER && o.precision != GAHHG_QUERY_FP64_FILTER)) {
        set_error("gahhg_server_create: invalid options");
        return GAHHG_ERR_ARG;
    }
    if (o.direct_min_points < 1) o.direct_min_points = 1;
    gahhg_server* s = new gahhg_server();
    s->o = o;
    const gahhg_status st = s->init();
    if (st != GAHHG_OK) {
        const std::string msg = last_error();
        delete s;
        set_error("gahhg_server_create: %s", msg.c_str());
        return st;
    }
    *out = s;
    return GAHHG_OK;
}

gahhg_status gahhg_server_submit_build(gahhg_server* s, const gahhg_polygon* poly, int top_cells, int leaf_edges,
                                       int flags, int* id, int64_t* ticket)
{
    if (!s || !poly || poly->p.pv_num <= 0) {
        set_error("submit_build: need a server and a polygon with edges");
        return GAHHG_ERR_ARG;
    }
    auto copy = std::make_unique<Polygon>();
    copy->copy_host(poly->p);
    const long long edges = copy->pv_num;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->broken) {
        set_error("server stopped after a device error: %s", s->broken_msg.c_str());
        return GAHHG_ERR_CUDA;
    }
    int pid;
    if (!s->free_ids.empty()) {
        pid = s->free_ids.back();
        s->free_ids.pop_back();
    } else if (s->next_id < s->o.max_polygons) {
        pid = s->next_id++;
    } else {
        set_error("submit_build: all %d polygon ids are in use", s->o.max_polygons);
        return GAHHG_ERR_CAPACITY;
    }
    SrvPoly& P = s->polys[pid];
    P = SrvPoly();
    P.poly = std::move(copy);
    P.state = GAHHG_POLY_QUEUED;
    P.top = top_cells;
    P.leaf = leaf_edges;
    P.pinned = (flags & GAHHG_SERVE_PINNED) != 0;
    P.est = s->estimate(edges);
    P.last_use = now_seconds();
    Req* r = new Req();
    r->build = true;
    r->poly = pid;
    r->detached = (flags & GAHHG_SERVE_DETACHED) != 0;
    r->t_submit = now_seconds();
    r->ticket = s->next_ticket++;
    P.build_req = r;
    if (!r->detached) s->tickets[r->ticket] = r;
    s->outstanding++;
    s->build_queue.push_back(pid);
    if (id) *id = pid;
    if (ticket) *ticket = r->ticket;
    s->cv_build.notify_all();
    return GAHHG_OK;
}

gahhg_status gahhg_server_submit_query(gahhg_server* s, int id, const double* lonlat, int64_t n, uint8_t* labels,
                                       int flags, int64_t* ticket)
{
    if (!s || n < 0 || (n > 0 && (!lonlat || !labels))) {
        set_error("submit_query: bad arguments");
        return GAHHG_ERR_ARG;
    }
    Req* r = new Req();
    r->t_submit = now_seconds();
    r->lonlat = lonlat;
    r->labels = labels;
    r->n = n;
    r->poly = id;
    r->detached = (flags & GAHHG_SERVE_DETACHED) != 0;
    if (n >= s->o.direct_min_points) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, lonlat) == cudaSuccess && a.type == cudaMemoryTypeHost) r->direct = true;
        cudaGetLastError();
        s->note_stall(STALL_POINTER_QUERY, r->t_submit, now_seconds());
    }
    const double tw = now_seconds();
    std::lock_guard<std::mutex> lk(s->mu);
    s->note_stall(STALL_SUBMIT_LOCK, tw, now_seconds());
    if (s->broken) {
        delete r;
        set_error("server stopped after a device error: %s", s->broken_msg.c_str());
        return GAHHG_ERR_CUDA;
    }
    if (id < 0 || id >= s->next_id) {
        delete r;
        set_error("submit_query: unknown polygon id %d", id);
        return GAHHG_ERR_ARG;
    }
    SrvPoly& P = s->polys[id];
    if (P.state != GAHHG_POLY_READY && P.state != GAHHG_POLY_QUEUED && P.state != GAHHG_POLY_BUILDING) {
        delete r;
        set_error("submit_query: polygon %d is not resident (state %d)", id, P.state);
        return GAHHG_ERR_ARG;
    }
    r->ticket = s->next_ticket++;
    if (ticket) *ticket = r->ticket;
    if (!r->detached) s->tickets[r->ticket] = r;
    s->outstanding++;
    P.refs++;
    if (n == 0) {
        s->complete_locked(r, GAHHG_OK);
        return GAHHG_OK;
    }
    if (P.state == GAHHG_POLY_READY) {
        s->pending.push_back(r);
        s->cv_dispatch.notify_one();
    } else {
        P.held.push_back(r);
    }
    return GAHHG_OK;
}

gahhg_status gahhg_server_wait(gahhg_server* s, int64_t ticket, double timeout_s)
{
    if (!s) return GAHHG_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) {
        set_error("wait: unknown ticket %lld", (long long)ticket);
        return GAHHG_ERR_ARG;
    }
    Req* r = it->second;
    if (!s->cv_wait.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return r->done; })) {
        set_error("wait: ticket %lld still pending", (long long)ticket);
        return GAHHG_ERR_STATE;
    }
    const gahhg_status st = r->status;
    if (st != GAHHG_OK) set_error("%s", r->msg.empty() ? "request failed" : r->msg.c_str());
    s->tickets.erase(ticket);
    delete r;
    return st;
}

gahhg_status gahhg_server_drain(gahhg_server* s, double timeout_s) { return s ? s->drain(timeout_s) : GAHHG_ERR_ARG; }

gahhg_status gahhg_server_evict(gahhg_server* s, int id)
{
    if (!s) return GAHHG_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    if (id >= 0 && id < s->next_id && s->polys[id].state == GAHHG_POLY_FAILED && s->polys[id].refs == 0) {
        s->polys[id].state = GAHHG_POLY_FREE;  // releases the id of a failed build
        s->free_ids.push_back(id);
        return GAHHG_OK;
    }
    if (id < 0 || id >= s->next_id || s->polys[id].state != GAHHG_POLY_READY) {
        set_error("evict: polygon %d is not resident", id);
        return GAHHG_ERR_ARG;
    }
    {
        SrvPoly& P = s->polys[id];
        if (P.refs == 0)
            s->free_poly_locked(id);
        else
            P.state = GAHHG_POLY_EVICTING;
    }
    return GAHHG_OK;
}

gahhg_status gahhg_server_polygon_state(gahhg_server* s, int id, int* state, long long* bytes)
{
    if (!s) return GAHHG_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (id < 0 || id >= s->o.max_polygons) {
        set_error("polygon id %d out of range", id);
        return GAHHG_ERR_ARG;
    }
    if (state) *state = id < s->next_id ? s->polys[id].state : GAHHG_POLY_FREE;
    if (bytes) *bytes = id < s->next_id ? s->polys[id].bytes : 0;
    return GAHHG_OK;
}

gahhg_status gahhg_server_stats_get(gahhg_server* s, gahhg_server_stats* out)
{
    if (!s || !out) return GAHHG_ERR_ARG;
    std::vector<double> lq, lb;
    gahhg_server_stats r;
    memset(&r, 0, sizeof(r));
    {
        std::lock_guard<std::mutex> lk(s->mu);
        lq = s->lat_q;
        lb = s->lat_b;
        r.queries_done = s->queries_done;
        r.query_points = s->query_points;
        r.builds_done = s->builds_done;
        r.builds_failed = s->builds_failed;
        r.evictions = s->evictions;
        r.batches = s->batches;
        r.pieces = s->pieces;
        r.resident_polygons = s->resident;
        r.pending_queries = (int)s->pending.size();
        r.pending_builds = (int)s->build_queue.size() + s->builds_running;
        r.inflight_batches = (int)s->inflight.size();
        r.resident_bytes = s->resident_bytes;
        r.hbm_budget = s->o.hbm_budget;
        r.window_s = now_seconds() - s->t0;
        r.mean_batch_points = s->batches ? (double)s->batch_points / (double)s->batches : 0.0;
        r.mean_batch_pieces = s->batches ? (double)s->pieces / (double)s->batches : 0.0;
        r.boundary_points = s->st_boundary;
        r.esc_fp64 = s->st_fp64;
        r.esc_exact = s->st_exact;
        r.in_count = s->st_in;
    }
    r.points_per_s = r.window_s > 0 ? (double)r.query_points / r.window_s : 0.0;
    r.p50_ms = percentile(lq, 0.50);
    r.p90_ms = percentile(lq, 0.90);
    r.p99_ms = percentile(lq, 0.99);
    r.max_ms = lq.empty() ? 0.0 : *std::max_element(lq.begin(), lq.end());
    r.build_p50_ms = percentile(lb, 0.50);
    r.build_p99_ms = percentile(lb, 0.99);
    *out = r;
    return GAHHG_OK;
}

gahhg_status gahhg_server_stats_reset(gahhg_server* s)
{
    if (!s) return GAHHG_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    s->lat_q.clear();
    s->lat_b.clear();
    s->trace.clear();
    {
        std::lock_guard<std::mutex> lk2(s->stall_mu);
        s->stalls.clear();
    }
    s->queries_done = s->query_points = s->builds_done = s->builds_failed = s->evictions = 0;
    s->batches = s->pieces = s->batch_points = 0;
    s->st_boundary = s->st_fp64 = s->st_exact = s->st_in = 0;
    s->t0 = now_seconds();
    return GAHHG_OK;
}

long long gahhg_server_latencies(gahhg_server* s, int kind, double* out, long long cap)
{
    if (!s) return 0;
    std::lock_guard<std::mutex> lk(s->mu);
    const std::vector<double>& v = kind == 1 ? s->lat_b : s->lat_q;
    if (out)
        for (long long i = 0; i < std::min<long long>(cap, (long long)v.size()); i++) out[i] = v[i];
    return (long long)v.size();
}

long long gahhg_server_trace(gahhg_server* s, double* out, long long cap)
{
    if (!s) return 0;
    std::lock_guard<std::mutex> lk(s->mu);
    if (out)
        for (long long i = 0; i < std::min<long long>(cap, (long long)s->trace.size()); i++)
            memcpy(out + 6 * i, s->trace[i].data(), 6 * sizeof(double));
    return (long long)s->trace.size();
}

long long gahhg_server_stalls(gahhg_server* s, double* out, long long cap)
{
    if (!s) return 0;
    std::lock_guard<std::mutex> lk(s->stall_mu);
    if (out)
        for (long long i = 0; i < std::min<long long>(cap, (long long)s->stalls.size()); i++)
            memcpy(out + 3 * i, s->stalls[i].data(), 3 * sizeof(double));
    return (long long)s->stalls.size();
}

void gahhg_server_free(gahhg_server* s)
{
    if (!s) return;
    s->drain(60.0);
    delete s;
}

}  // extern "C"
