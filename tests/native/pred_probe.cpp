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
