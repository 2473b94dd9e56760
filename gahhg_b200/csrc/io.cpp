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
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cfloat>
#include <fstream>
#include <sstream>

#include "gahhg_canon.h"
#include "gahhg_internal.h"

namespace gahhg {

namespace {

bool read_file(const char* path, std::string* out)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    std::ostringstream ss;
    ss << f.rdbuf();
    *out = ss.str();
    return true;
}

// Splits into lines the way repeated istream::getline does: '\n' ends a line
// and is dropped; a final line without '\n' still counts; nothing after the
// last '\n' means no further line.
struct LineReader {
    const std::string& s;
    size_t pos = 0;
    explicit LineReader(const std::string& str) : s(str) {}
    // returns false at end of data (getline would fail); *line = "" then
    bool next(std::string* line)
    {
        if (pos >= s.size()) {
            line->clear();
            return false;
        }
        size_t e = s.find('\n', pos);
        if (e == std::string::npos) e = s.size();
        line->assign(s, pos, e - pos);
        pos = (e < s.size()) ? e + 1 : e;
        return true;
    }
};

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

// Builds pv and pe from ring vertex lists (closing vertices already removed).
void assemble(Polygon* P)
{
    const int nr = P->num_rings;
    P->pv_num = P->ring_start[nr];
    P->pv.resize(P->pv_num);
    for (int i = 0; i < P->pv_num; i++) P->pv[i] = vertex_xyz(P->lonlat[2 * i], P->lonlat[2 * i + 1]);
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

// `sscanf(buf, "%lf %lf", &lo, &la) == 2` with the same acceptance.
bool parse_two(const std::string& line, double* lo, double* la)
{
    return sscanf(line.c_str(), "%lf %lf", lo, la) == 2;
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
    LineReader rd(data);
    std::string line;
    int lineindex = 0;
    auto fail_format = [&](const char* what) {
        printf("Error. Line %d of %s. %s\n", lineindex, path, what);
        set_error("line %d of %s: %s", lineindex, path, what);
        return GAHHG_ERR_FORMAT;
    };
    const char* WRONG = "Wrong format.";
    const char* FEW = "Number of edges should be greater than 3. ";

    int inNum = 0, outVNum = 0, temp = 0;
    rd.next(&line);
    lineindex++;
    if (sscanf(line.c_str(), "POLYGON 1 %d", &inNum) != 1) return fail_format(WRONG);
    rd.next(&line);
    lineindex++;
    if (sscanf(line.c_str(), "0 %d", &outVNum) != 1) return fail_format(WRONG);
    if (outVNum < 4) return fail_format(FEW);

    std::vector<std::vector<double>> rings;
    rings.emplace_back();
    for (int i = 0; i < outVNum; i++) {
        rd.next(&line);
        lineindex++;
        double lo, la;
        if (!parse_two(line, &lo, &la)) return fail_format(WRONG);
        if (i < outVNum - 1) {
            rings[0].push_back(lo);
            rings[0].push_back(la);
        }
    }
    for (int h = 0; h < inNum; h++) {
        rd.next(&line);
        lineindex++;
        int nv = 0;
        if (sscanf(line.c_str(), "%d %d", &temp, &nv) != 2) return fail_format(WRONG);
        if (nv < 4) return fail_format(FEW);
        rings.emplace_back();
        for (int j = 0; j < nv; j++) {
            rd.next(&line);
            lineindex++;
            double lo, la;
            if (!parse_two(line, &lo, &la)) return fail_format(WRONG);
            if (j < nv - 1) {
                rings.back().push_back(lo);
                rings.back().push_back(la);
            }
        }
    }
    P->path = path;
    P->num_rings = (int)rings.size();
    P->ring_start.assign(1, 0);
    P->lonlat.clear();
    for (auto& r : rings) {
        P->lonlat.insert(P->lonlat.end(), r.begin(), r.end());
        P->ring_start.push_back(P->ring_start.back() + (int)(r.size() / 2));
    }
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

gahhg_status load_points_file(const char* path, Points* T)
{
    printf("Load test points from a CSV file: %s.\n", path);
    std::string data;
    if (!read_file(path, &data)) {
        printf("Error. Can not open %s\n.", path);
        set_error("cannot open %s", path);
        return GAHHG_ERR_IO;
    }
    T->lonlat.clear();
    T->lonlat.reserve(data.size() / 10);
    const char* s = data.c_str();
    const char* end = s + data.size();
    long long count = 0;
    while (s < end) {
        const char* e = (const char*)memchr(s, '\n', end - s);
        if (!e) e = end;
        // "%lf,%lf": optional white space, number, ',', optional white space, number
        char* q;
        const char* p = s;
        double lo = strtod(p, &q);
        bool ok = q != p && q < e;
        double la = 0;
        if (ok) {
            ok = (*q == ',');
            if (ok) {
                p = q + 1;
                la = strtod(p, &q);
                ok = q != p && q <= e;
            }
        }
        if (!ok) {
            printf("Error. Line %lld of %s. Wrong format.\n", count + 1, path);
            set_error("line %lld of %s: wrong format", count + 1, path);
            return GAHHG_ERR_FORMAT;
        }
        T->lonlat.push_back(lo);
        T->lonlat.push_back(la);
        count++;
        s = (e < end) ? e + 1 : e;
    }
    T->path = path;
    return GAHHG_OK;
}

}  // namespace gahhg
