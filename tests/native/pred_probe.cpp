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
// kernel runs it, with the edge record built as the index build builds it.
// Per case (8 doubles): query lon, lat (raw; the FakeLL round trip is applied
// here), center lon, lat, then A lon, lat and B lon, lat.  out: s2, s3, s4
// (0 = undecided), or 9 9 9 when the offset is not small.
#include "../../gahhg_b200/csrc/local_frame.cuh"

extern "C" void local_signs(const double* cfg, long n, int* out)
{
    using namespace gahhg;
    for (long i = 0; i < n; i++) {
        const double* c = cfg + 8 * i;
        double R[3], A[3], B[3], n1[3], n2[3], n3[3];
        gahhg_canon_vertex_xyz(c[2], c[3], R);
        gahhg_canon_vertex_xyz(c[4], c[5], A);
        gahhg_canon_vertex_xyz(c[6], c[7], B);
        exact::cross_value(A, B, n1);
        exact::cross_value(A, R, n2);
        exact::cross_value(B, R, n3);
        float f1[3], f2[3], f3[3];
        for (int j = 0; j < 3; j++) {
            f1[j] = (float)n1[j];
            f2[j] = (float)n2[j];
            f3[j] = (float)n3[j];
        }
        const float h1 = (float)exact::det3_value(A, B, R);
        local_frame::Offset o;
        int* s = out + 3 * i;
        if (!local_frame::offset(c[0], gahhg_canon_query_lat(c[1]), c[2], c[3], o)) {
            s[0] = s[1] = s[2] = 9;
            continue;
        }
        s[0] = local_frame::sign_at(o, f1, h1);
        s[1] = local_frame::sign_at(o, f2, 0.0f);
        s[2] = local_frame::sign_at(o, f3, 0.0f);
    }
}
