// Host build of the FP64 filters of gahhg_b200/csrc/exact_pred.cuh, for the
// CPU soundness test (tests/test_cpu_predicates.py): out[i] = filter sign of
// the triple (a, b, c) at rows 3i, 3i+1, 3i+2 of xyz (0 = undecided).
#include "../../gahhg_b200/csrc/exact_pred.cuh"

extern "C" void filter_signs(const double* xyz, long n, int near, int* out)
{
    for (long i = 0; i < n; i++) {
        const double* a = xyz + 9 * i;
        out[i] = near ? gahhg::exact::orient_fp64_near(a, a + 3, a + 6) : gahhg::exact::orient_fp64(a, a + 3, a + 6);
    }
}

// The FP32 local-frame tier (gahhg_b200/csrc/local_frame.cuh) as the query
// kernel runs it, with the edge record built as the index build builds it
// (ends in the order that makes orient(A, B, R) = +1).  Per case (8
// doubles): query lon, lat (raw; the FakeLL round trip is applied here),
// center lon, lat, then A lon, lat and B lon, lat.  out: s2 = orient(A, B, q),
// s3 = orient(R, q, A), s4 = orient(R, q, B) in the given order of A and B
// (0 = undecided), then the tier's crossing test of the record (1 crossing,
// 0 none, -1 undecided), or 9 9 9 9 when the offset is not small.
#include "../../gahhg_b200/csrc/local_frame.cuh"

extern "C" void local_signs(const double* cfg, long n, int* out)
{
    using namespace gahhg;
    for (long i = 0; i < n; i++) {
        const double* c = cfg + 8 * i;
        double R[3], A[3], B[3];
        gahhg_canon_vertex_xyz(c[2], c[3], R);
        gahhg_canon_vertex_xyz(c[4], c[5], A);
        gahhg_canon_vertex_xyz(c[6], c[7], B);
        const int s1 = exact::orient(A, B, R);
        const bool swap = s1 < 0;
        float r[4];
        local_frame::Basis fb;
        local_frame::basis_at(c[2], c[3], fb);
        local_frame::edge_record(A, B, fb, swap, r);
        // the leaf record's sine and cosine of the center's canonical latitude
        double sb, cb;
        gahhg_canon_sincos(gahhg_canon_rad(c[3]), &sb, &cb);
        local_frame::Frame f;
        int* s = out + 4 * i;
        if (s1 == 0 || !(fabs(c[0]) <= 540.0) ||
            !local_frame::frame_at(c[0], gahhg_canon_query_lat(c[1]), c[2], c[3], (float)sb, (float)cb, f)) {
            s[0] = s[1] = s[2] = s[3] = 9;
            continue;
        }
        local_frame::Tests t;
        local_frame::tests_of(f, t);
        const int e = local_frame::sign_edge(t, r[0], r[1], r[2], r[3]);
        const int ea = local_frame::sign_end(t, r[0], r[1]), eb = local_frame::sign_end(t, r[2], r[3]);
        s[0] = swap ? -e : e;
        s[1] = swap ? eb : ea;
        s[2] = swap ? ea : eb;
        // the tier's combined test, on the stored order
        s[3] = local_frame::record_crossing(t, r[0], r[1], r[2], r[3]);
    }
}

// The kernels' exact predicate for the rational-arithmetic test
// (tests/test_cpu_oracle_exact_sign.py): out[2i] = the exact sign of
// det[a; b; c] by expansions (stage 2, 0 when it vanishes), out[2i+1] =
// orient (stages 1-3, simulation of simplicity for a vanishing determinant).
extern "C" void exact_signs(const double* xyz, long n, int* out)
{
    for (long i = 0; i < n; i++) {
        const double* a = xyz + 9 * i;
        out[2 * i] = gahhg::exact::det3_sign(a, a + 3, a + 6);
        out[2 * i + 1] = gahhg::exact::orient(a, a + 3, a + 6);
    }
}
