// io.cpp - POLYGON and CSV loaders, result writer.
//
// Loader behaviour follows the reference:
//   GPISPPolygon::loadPolyFromTXT  source/GPISPPolygon.cu:32-278
//   GPISPPolygon::isPolyClockwise  source/GPISPPolygon.cu:280-313
//   GPISPTP::loadTPFromCSV         source/GPISPTP.cu:13-79
//   GPISPTP::exportResult2CSV      source/GPISPTP.cu:81-99
// Same accepted syntax (the same sscanf formats), the same messages on stdout,
// the same failure points; the closing vertex of every ring is dropped; the
// outer ring is re-oriented counter-clockwise and holes clockwise by the
// reference's local test at the northernmost vertex.  Vertex XYZ comes from
// the canonical conversion (include/gahhg_canon.h).
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cfloat>
#include <charconv>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <climits>
#include <cmath>
#include <mutex>
#include <thread>
#include <vector>

#include "gahhg_canon.h"
#include "gahhg_internal.h"

namespace gahhg {

namespace {

// The whole file in one read into a string sized from fstat.
bool read_file(const char* path, std::string* out)
{
    FILE* f = fopen(path, "rb");
    if (!f) return false;
    struct stat st;
    if (fstat(fileno(f), &st) != 0 || !S_ISREG(st.st_mode)) {
        fclose(f);
        return false;
    }
    out->resize((size_t)st.st_size);
    const size_t got = st.st_size ? fread(&(*out)[0], 1, (size_t)st.st_size, f) : 0;
    fclose(f);
    out->resize(got);
    return true;
}

D3 vertex_xyz(double lon, double lat)
{
    double p[3];
    gahhg_canon_vertex_xyz(lon, lat, p);
    return d3(p[0], p[1], p[2]);
}

// isPolyClockwise (source/GPISPPolygon.cu:280-313): orientation from the
// northernmost vertex (first one on ties) and its two neighbours.
bool ring_clockwise(const double* lonlat, int n)
{
    double maxvalue = -FLT_MAX;
    int maxindex = 0;
    for (int i = 0; i < n; i++) {
        if (lonlat[2 * i + 1] > maxvalue) {
            maxvalue = lonlat[2 * i + 1];
            maxindex = i;
        }
    }
    const int ip = (maxindex == 0) ? n - 1 : maxindex - 1;
    const int in = (maxindex == n - 1) ? 0 : maxindex + 1;
    D3 a0 = vertex_xyz(lonlat[2 * ip], lonlat[2 * ip + 1]);
    D3 a1 = vertex_xyz(lonlat[2 * maxindex], lonlat[2 * maxindex + 1]);
    D3 b = vertex_xyz(lonlat[2 * in], lonlat[2 * in + 1]);
    D3 e = a1 - a0;
    D3 nn = normalize(cross(a0, e));
    double temp = dot(nn, b);
    return !(temp > 0);
}

// `sscanf(buf, "%lf %lf", &lo, &la) == 2` with the same acceptance.
bool parse_two(const std::string& line, double* lo, double* la)
{
    return sscanf(line.c_str(), "%lf %lf", lo, la) == 2;
}

inline bool poly_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

// A plain decimal number at p (sign '-' or none): the cases where
// std::from_chars and the reference's "%lf" read the same characters to the
// same (correctly rounded) value.  False leaves the line to sscanf.
inline bool plain_number(const char* p, const char* e, double* v, const char** end)
{
    if (p >= e || !((*p >= '0' && *p <= '9') || *p == '-' || *p == '.')) return false;
    const auto r = std::from_chars(p, e, *v);
    if (r.ec != std::errc() || !std::isfinite(*v)) return false;
    // an exponent or hex marker that from_chars stopped before may be read
    // differently by scanf (which cannot back out of "1e")
    if (r.ptr < e && (*r.ptr == 'e' || *r.ptr == 'E' || *r.ptr == 'x' || *r.ptr == 'X')) return false;
    *end = r.ptr;
    return true;
}

// "%lf %lf" on line [s, e): the usual "lon lat" by from_chars, anything else
// (a '+' sign, hex, inf/nan, no white space between the numbers, a second
// number missing) by sscanf itself on a NUL-terminated copy.
bool parse_two_line(const char* s, const char* e, double* lo, double* la)
{
    const char* p = s;
    while (p < e && poly_space(*p)) p++;
    const char* q;
    if (plain_number(p, e, lo, &q) && q < e && poly_space(*q)) {
        p = q;
        while (p < e && poly_space(*p)) p++;
        if (plain_number(p, e, la, &q)) return true;
    }
    return parse_two(std::string(s, e), lo, la);
}

// Vertex XYZ of points [a, b) of P (canonical conversion).
void vertex_range(Polygon* P, int a, int b)
{
    for (int i = a; i < b; i++) P->pv[i] = vertex_xyz(P->lonlat[2 * i], P->lonlat[2 * i + 1]);
}

// Splits [0, n) into up to `hw` ranges of at least `grain` items and runs
// f(a, b) on each, the first on the calling thread.
template <class F>
void parallel_ranges(long long n, long long grain, F f)
{
    const int hw = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const int nt = (int)std::max(1LL, std::min<long long>(hw, n / std::max(grain, 1LL)));
    if (nt == 1) {
        f(0LL, n);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 1; t < nt; t++) th.emplace_back(f, n * t / nt, n * (t + 1) / nt);
    f(0LL, n / nt);
    for (auto& x : th) x.join();
}

// Builds pv and pe from ring vertex lists (closing vertices already removed).
void assemble(Polygon* P)
{
    const int nr = P->num_rings;
    P->pv_num = P->ring_start[nr];
    P->pv.resize(P->pv_num);
    parallel_ranges(P->pv_num, 1 << 16, [P](long long a, long long b) { vertex_range(P, (int)a, (int)b); });
    P->pe.assign(2 * (size_t)P->pv_num, 0);
    int index = 0;
    for (int r = 0; r < nr; r++) {
        const int start = P->ring_start[r];
        const int m = P->ring_start[r + 1] - start;
        bool cw = ring_clockwise(&P->lonlat[2 * (size_t)start], m);
        // outer ring must run counter-clockwise, holes clockwise (:209-215)
        bool reverse = (r == 0) ? cw : !cw;
        if (!reverse) {
            for (int j = 0; j < m; j++) {
                P->pe[2 * index] = index;
                P->pe[2 * index + 1] = index + 1;
                index++;
            }
            P->pe[2 * index - 1] = start;
        } else {
            for (int j = m - 1; j >= 0; j--) {
                P->pe[2 * index] = start + j;
                P->pe[2 * index + 1] = start + j - 1;
                index++;
            }
            P->pe[2 * index - 1] = start + m - 1;
        }
    }
}

}  // namespace

gahhg_status load_polygon_file(const char* path, Polygon* P)
{
    printf("Load spherical polygon from %s.\n", path);
    std::string data;
    if (!read_file(path, &data)) {
        printf("Error. Can not open %s\n.", path);
        set_error("cannot open %s", path);
        return GAHHG_ERR_IO;
    }
    const char* WRONG = "Wrong format.";
    const char* FEW = "Number of edges should be greater than 3. ";
    // Lines as repeated getline sees them: '\n' ends a line; a final line
    // without '\n' counts; reading past the last line gives "".
    std::vector<size_t> start;
    start.reserve(data.size() / 16 + 2);
    for (size_t pos = 0; pos < data.size();) {
        start.push_back(pos);
        const void* nl = memchr(data.data() + pos, '\n', data.size() - pos);
        pos = nl ? (size_t)((const char*)nl - data.data()) + 1 : data.size();
    }
    const long long nlines = (long long)start.size();
    auto line_begin = [&](long long k) { return data.data() + start[k]; };
    auto line_end = [&](long long k) {
        const size_t e = (k + 1 < nlines) ? start[k + 1] - 1 : data.size();
        return data.data() + ((e > start[k] && data[e - 1] == '\n') ? e - 1 : e);
    };
    // The reference reads each line with getline(buf, size), size = the
    // file's size, which stores at most size - 1 characters: only a file that
    // is a single line without '\n' reaches that, and it loses its last
    // character (the stream then fails, so later lines read as "").
    const bool cut_last = nlines == 1 && !data.empty() && data.back() != '\n';
    auto line_str = [&](long long k) {
        if (k >= nlines) return std::string();
        std::string s(line_begin(k), line_end(k));
        if (cut_last && !s.empty()) s.pop_back();
        return s;
    };
    // The first failing line (1-based, as the reference counts) and its message.
    long long fail_line = LLONG_MAX;
    const char* fail_what = nullptr;
    auto note = [&](long long line, const char* what) {
        if (line < fail_line) {
            fail_line = line;
            fail_what = what;
        }
    };

    // The structure (ring headers and the vertex blocks they announce) is
    // read serially; vertex lines are parsed afterwards, in parallel.
    struct Block {
        long long first;  // 0-based line of the ring's first vertex
        int nv;           // vertex lines announced (the last closes the ring)
    };
    std::vector<Block> blocks;
    int inNum = 0, outVNum = 0, temp = 0;
    long long k = 0;
    if (sscanf(line_str(k).c_str(), "POLYGON 1 %d", &inNum) != 1) {
        note(k + 1, WRONG);
    } else if (sscanf(line_str(k + 1).c_str(), "0 %d", &outVNum) != 1) {
        note(k + 2, WRONG);
    } else if (outVNum < 4) {
        note(k + 2, FEW);
    } else {
        k = 2;
        blocks.push_back({k, outVNum});
        k += outVNum;
        for (int h = 0; h < inNum && k <= nlines; h++) {
            int nv = 0;
            if (sscanf(line_str(k).c_str(), "%d %d", &temp, &nv) != 2) {
                note(k + 1, WRONG);
                break;
            }
            if (nv < 4) {
                note(k + 1, FEW);
                break;
            }
            blocks.push_back({k + 1, nv});
            k += 1 + (long long)nv;
        }
    }
    // vertex lines beyond the end of the file read as "": the first fails
    std::vector<long long> vfirst(blocks.size() + 1, 0);  // flattened vertex index of each block
    for (size_t r = 0; r < blocks.size(); r++) {
        long long have = std::max(0LL, std::min<long long>(blocks[r].nv, nlines - blocks[r].first));
        if (have < blocks[r].nv) note(blocks[r].first + have + 1, WRONG);
        vfirst[r + 1] = vfirst[r] + have;
    }
    // (announced counts may be absurd in a truncated file: 64-bit sums, and
    // vertex storage only once every announced line is present)
    std::vector<long long> ring_start(1, 0);
    for (const Block& bl : blocks) ring_start.push_back(ring_start.back() + bl.nv - 1);
    std::vector<double> lonlat;
    if (fail_line == LLONG_MAX) {
        if (ring_start.back() > INT_MAX / 2) {
            set_error("%s: %lld vertices exceed the loader's limit", path, ring_start.back());
            return GAHHG_ERR_CAPACITY;
        }
        lonlat.resize(2 * (size_t)ring_start.back());
    }
    std::mutex mu;
    parallel_ranges(vfirst.back(), 1 << 15, [&](long long a, long long b) {
        long long bad = LLONG_MAX;
        size_t r = std::upper_bound(vfirst.begin(), vfirst.end(), a) - vfirst.begin() - 1;
        for (long long v = a; v < b; v++) {
            while (v >= vfirst[r + 1]) r++;
            const long long j = v - vfirst[r];
            const long long ln = blocks[r].first + j;
            double lo, la;
            if (!parse_two_line(line_begin(ln), line_end(ln), &lo, &la)) {
                bad = std::min(bad, ln + 1);
                continue;
            }
            if (j < blocks[r].nv - 1 && !lonlat.empty()) {
                const size_t at = 2 * ((size_t)ring_start[r] + (size_t)j);
                lonlat[at] = lo;
                lonlat[at + 1] = la;
            }
        }
        if (bad != LLONG_MAX) {
            std::lock_guard<std::mutex> lock(mu);
            note(bad, WRONG);
        }
    });
    if (fail_line != LLONG_MAX) {
        printf("Error. Line %lld of %s. %s\n", fail_line, path, fail_what);
        set_error("line %lld of %s: %s", fail_line, path, fail_what);
        return GAHHG_ERR_FORMAT;
    }
    P->path = path;
    P->num_rings = (int)blocks.size();
    P->ring_start.assign(ring_start.begin(), ring_start.end());
    P->lonlat = std::move(lonlat);
    assemble(P);
    return GAHHG_OK;
}

gahhg_status polygon_from_rings(const double* lonlat, const int64_t* ring_offsets, int nrings, Polygon* P)
{
    if (!lonlat || !ring_offsets || nrings < 1) {
        set_error("polygon_from_rings: need at least one ring");
        return GAHHG_ERR_ARG;
    }
    P->num_rings = nrings;
    P->ring_start.assign(1, 0);
    P->lonlat.clear();
    for (int r = 0; r < nrings; r++) {
        int64_t a = ring_offsets[r], b = ring_offsets[r + 1];
        if (b - a < 3) {
            set_error("ring %d has %lld vertices; at least 3 are needed", r, (long long)(b - a));
            return GAHHG_ERR_FORMAT;
        }
        P->lonlat.insert(P->lonlat.end(), lonlat + 2 * a, lonlat + 2 * b);
        P->ring_start.push_back(P->ring_start.back() + (int)(b - a));
    }
    P->path = "<memory>";
    assemble(P);
    return GAHHG_OK;
}

namespace {

// Read-only map of a whole file (an empty file maps to nothing).
struct MappedFile {
    const char* data = nullptr;
    size_t size = 0;
    struct stat st {};
    int fd = -1;
    bool open(const char* path)
    {
        fd = ::open(path, O_RDONLY);
        if (fd < 0 || fstat(fd, &st) != 0 || !S_ISREG(st.st_mode)) return false;
        size = (size_t)st.st_size;
        if (size == 0) return true;
        void* p = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
        if (p == MAP_FAILED) return false;
        madvise(p, size, MADV_SEQUENTIAL);
        data = (const char*)p;
        return true;
    }
    ~MappedFile()
    {
        if (data) munmap((void*)data, size);
        if (fd >= 0) ::close(fd);
    }
};

inline bool in_line_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f'; }

// The reference's reading of one line [s, e): sscanf(line, "%lf,%lf") of the
// platform's C library, as GPISPTP::loadTPFromCSV does (source/GPISPTP.cu:
// 36), on a NUL-terminated copy of the line.  (glibc's %lf takes the digits
// of a number whose exponent has no digits, "1e,2" -> 1, 2, where strtod
// would stop before the 'e'; reading through sscanf keeps the reference's
// answer on every such line.)
bool parse_point_scanf(const char* s, const char* e, double* lo, double* la)
{
    char small[256];
    std::string big;
    char* buf = small;
    const size_t len = (size_t)(e - s);
    if (len + 1 > sizeof(small)) {
        big.assign(s, len);
        buf = &big[0];
    } else {
        memcpy(small, s, len);
        small[len] = 0;
    }
    return sscanf(buf, "%lf,%lf", lo, la) == 2;
}

// Fast path for the usual "lon,lat" line; false sends the line to the
// reading above (a '+' sign, hex, out-of-range values, an exponent without
// digits, unusual separators).
inline bool parse_point_fast(const char* s, const char* e, double* lo, double* la)
{
    const char* p = s;
    while (p < e && in_line_space(*p)) p++;
    auto r = std::from_chars(p, e, *lo);
    if (r.ec != std::errc() || r.ptr >= e || *r.ptr != ',') return false;
    p = r.ptr + 1;
    while (p < e && in_line_space(*p)) p++;
    r = std::from_chars(p, e, *la);
    if (r.ec != std::errc()) return false;
    return r.ptr == e || in_line_space(*r.ptr) || *r.ptr == ',' || *r.ptr == ';';
}

// Lines of [b, e) that start a line (b is a line start): '\n' ends a line; a
// final line without '\n' counts when this chunk ends the file.
long long count_lines(const char* b, const char* e, bool last)
{
    long long n = (long long)std::count(b, e, '\n');
    if (last && e > b && e[-1] != '\n') n++;
    return n;
}

constexpr uint64_t SIDECAR_MAGIC = 0x3146545032474847ull;  // "GHG2PTF1"

struct SidecarHeader {
    uint64_t magic;
    uint64_t count;
    uint64_t source_size;
    int64_t source_mtime_ns;
    uint64_t reserved[4];
};
static_assert(sizeof(SidecarHeader) == 64, "sidecar header");

std::string sidecar_path(const char* csv) { return std::string(csv) + ".f64"; }

int64_t mtime_ns(const struct stat& st) { return (int64_t)st.st_mtim.tv_sec * 1000000000LL + st.st_mtim.tv_nsec; }

}  // namespace

// GPISPTP::loadTPFromCSV (source/GPISPTP.cu:13-79).  The file is mapped and
// split at line starts into one chunk per host thread; a first pass counts
// each chunk's lines, a second parses them in place.  Values and the first
// rejected line (and its message) are those of the reference's serial
// sscanf("%lf,%lf") reading.
gahhg_status load_points_file(const char* path, Points* T)
{
    printf("Load test points from a CSV file: %s.\n", path);
    MappedFile f;
    if (!f.open(path)) {
        printf("Error. Can not open %s\n.", path);
        set_error("cannot open %s", path);
        return GAHHG_ERR_IO;
    }
    const char* base = f.data;
    const char* end = base + f.size;
    // The reference reads each line with getline(buf, size), size = the
    // file's size, which stores at most size - 1 characters: a non-empty file
    // without any '\n' (one line, no line end) fails on its first line, and
    // the reference's loop stops there with no points and no error.
    if (f.size > 0 && !memchr(base, '\n', f.size)) {
        T->lonlat.reset();
        T->n = 0;
        T->path = path;
        return GAHHG_OK;
    }
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const int nt = (int)std::min<size_t>(std::min(hw, 64u), std::max<size_t>(1, f.size >> 22));  // >= 4 MB each
    std::vector<const char*> cut(nt + 1);
    cut[0] = base;
    cut[nt] = end;
    for (int t = 1; t < nt; t++) {
        const char* c = base + f.size / nt * t;
        c = std::max(c, cut[t - 1]);
        const char* nl = c < end ? (const char*)memchr(c, '\n', end - c) : nullptr;
        cut[t] = nl ? nl + 1 : end;
    }
    std::vector<long long> first(nt + 1, 0);
    auto run = [&](auto&& fn) {
        if (nt == 1) {
            fn(0);
            return;
        }
        std::vector<std::thread> th;
        for (int t = 0; t < nt; t++) th.emplace_back(fn, t);
        for (auto& x : th) x.join();
    };
    run([&](int t) { first[t + 1] = count_lines(cut[t], cut[t + 1], t == nt - 1); });
    for (int t = 0; t < nt; t++) first[t + 1] += first[t];
    const long long n = first[nt];
    T->lonlat.reset(n ? new double[(size_t)n * 2] : nullptr);
    T->n = 0;
    std::vector<long long> bad(nt, -1);  // first rejected line (global index) per chunk
    run([&](int t) {
        double* out = T->lonlat.get() + 2 * first[t];
        const char* s = cut[t];
        const char* ce = cut[t + 1];
        long long k = 0;
        while (s < ce) {
            const char* e = (const char*)memchr(s, '\n', ce - s);
            if (!e) e = ce;
            double lo, la;
            if (!parse_point_fast(s, e, &lo, &la) && !parse_point_scanf(s, e, &lo, &la)) {
                bad[t] = first[t] + k;
                return;
            }
            out[2 * k] = lo;
            out[2 * k + 1] = la;
            k++;
            s = (e < ce) ? e + 1 : e;
        }
    });
    for (int t = 0; t < nt; t++)
        if (bad[t] >= 0) {
            printf("Error. Line %lld of %s. Wrong format.\n", bad[t] + 1, path);
            set_error("line %lld of %s: wrong format", bad[t] + 1, path);
            T->lonlat.reset();
            return GAHHG_ERR_FORMAT;
        }
    T->n = (size_t)n;
    T->path = path;
    return GAHHG_OK;
}

gahhg_status load_points_sidecar(const char* csv_path, Points* T)
{
    struct stat src;
    if (stat(csv_path, &src) != 0) {
        set_error("cannot open %s", csv_path);
        return GAHHG_ERR_IO;
    }
    const std::string sp = sidecar_path(csv_path);
    MappedFile f;
    if (!f.open(sp.c_str()) || f.size < sizeof(SidecarHeader)) {
        set_error("no sidecar %s", sp.c_str());
        return GAHHG_ERR_STATE;
    }
    SidecarHeader h;
    memcpy(&h, f.data, sizeof(h));
    if (h.magic != SIDECAR_MAGIC || h.source_size != (uint64_t)src.st_size || h.source_mtime_ns != mtime_ns(src) ||
        f.size != sizeof(h) + h.count * 16) {
        set_error("sidecar %s does not match %s", sp.c_str(), csv_path);
        return GAHHG_ERR_STATE;
    }
    T->lonlat.reset(h.count ? new double[h.count * 2] : nullptr);
    if (h.count) memcpy(T->lonlat.get(), f.data + sizeof(h), h.count * 16);
    T->n = h.count;
    T->path = csv_path;
    return GAHHG_OK;
}

gahhg_status write_points_sidecar(const char* csv_path, const Points& T)
{
    struct stat src;
    if (stat(csv_path, &src) != 0) {
        set_error("cannot open %s", csv_path);
        return GAHHG_ERR_IO;
    }
    const std::string sp = sidecar_path(csv_path);
    const std::string tmp = sp + ".tmp";
    FILE* fp = fopen(tmp.c_str(), "wb");
    if (!fp) {
        set_error("cannot write %s", tmp.c_str());
        return GAHHG_ERR_IO;
    }
    SidecarHeader h{};
    h.magic = SIDECAR_MAGIC;
    h.count = T.n;
    h.source_size = (uint64_t)src.st_size;
    h.source_mtime_ns = mtime_ns(src);
    bool ok = fwrite(&h, sizeof(h), 1, fp) == 1;
    if (ok && T.n) ok = fwrite(T.lonlat.get(), 16, T.n, fp) == T.n;
    ok = (fclose(fp) == 0) && ok;
    if (!ok || rename(tmp.c_str(), sp.c_str()) != 0) {
        unlink(tmp.c_str());
        set_error("cannot write %s", sp.c_str());
        return GAHHG_ERR_IO;
    }
    return GAHHG_OK;
}

}  // namespace gahhg
