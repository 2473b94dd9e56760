// cli.cpp - `gahhg`, the drop-in for GPISP.exe (source/GPISP.cu:15-70).
//
// Same flags (/polyfile /tpfile /reportfile /resultfile, unknown flags
// skipped), same defaults (source/GPISPParam.h:64-77), same messages, same
// return codes (-1 when a loader fails), the report block appended and the
// result CSV overwritten.  Extra flags: /maxdepth N, /semantics exact|reference
// (default reference, as GPISP.exe), /precision fp32|fp64, /sidecar (binary copy
// of the query file, `<tpfile>.f64`, read when it matches the CSV).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "gahhg.h"

int main(int argc, char* argv[])
{
    std::string poly = "NA0.txt", tp = "NA_query.csv", report = "report.txt", result = "result.csv";
    gahhg_build_opts o;
    gahhg_build_opts_init(&o);
    o.semantics = GAHHG_SEMANTICS_REFERENCE;
    o.verbose = 1;
    int precision = GAHHG_QUERY_AUTO;
    int point_flags = 0;
    for (int i = 1; i < argc; i++) {
        auto val = [&](std::string* dst) {
            if (i + 1 < argc) *dst = argv[++i];
        };
        if (!strcmp(argv[i], "/polyfile")) val(&poly);
        else if (!strcmp(argv[i], "/reportfile")) val(&report);
        else if (!strcmp(argv[i], "/resultfile")) val(&result);
        else if (!strcmp(argv[i], "/tpfile")) val(&tp);
        else if (!strcmp(argv[i], "/maxdepth") && i + 1 < argc) o.max_depth = atoi(argv[++i]);
        else if (!strcmp(argv[i], "/semantics") && i + 1 < argc) {
            const char* s = argv[++i];
            o.semantics = !strcmp(s, "exact") ? GAHHG_SEMANTICS_EXACT : GAHHG_SEMANTICS_REFERENCE;
        } else if (!strcmp(argv[i], "/precision") && i + 1 < argc) {
            const char* s = argv[++i];
            precision = !strcmp(s, "fp64") ? GAHHG_QUERY_FP64_FILTER : GAHHG_QUERY_FP32_FILTER;
        } else if (!strcmp(argv[i], "/sidecar")) {
            // read `<tpfile>.f64` when it matches the CSV, else parse and write it
            point_flags = GAHHG_POINTS_USE_SIDECAR | GAHHG_POINTS_WRITE_SIDECAR;
        }
    }
    gahhg_polygon* P = nullptr;
    if (gahhg_polygon_load(poly.c_str(), &P) != GAHHG_OK) return -1;
    gahhg_points* T = nullptr;
    if (gahhg_points_load_ex(tp.c_str(), point_flags, &T) != GAHHG_OK) return -1;
    gahhg_grid* G = nullptr;
    gahhg_status s = gahhg_build(P, &o, &G);
    if (s == GAHHG_OK) s = gahhg_classify(G);
    size_t n = gahhg_points_count(T);
    std::vector<uint8_t> labels(n);
    if (s == GAHHG_OK) s = gahhg_query(G, gahhg_points_lonlat(T), n, labels.data(), precision);
    if (s != GAHHG_OK) {
        fprintf(stderr, "gahhg: %s\n", gahhg_last_error());
        return 1;
    }
    gahhg_report_append(G, poly.c_str(), tp.c_str(), (long long)n, report.c_str(), 0);
    gahhg_result_write(result.c_str(), labels.data(), n);
    gahhg_grid_free(G);
    gahhg_points_free(T);
    gahhg_polygon_free(P);
    return 0;
}
