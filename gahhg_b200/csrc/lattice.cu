// lattice.cu - exact-semantics query index (placeholder until the exact engine lands).
#include "gahhg_internal.h"

namespace gahhg {
struct Lattice {
    int unused;
};
gahhg_status lattice_build(Grid* g)
{
    (void)g;
    return GAHHG_OK;
}
gahhg_status lattice_query(Grid*, const double*, size_t, uint8_t*, int, cudaStream_t, uint64_t*)
{
    set_error("exact engine not available");
    return GAHHG_ERR_STATE;
}
void lattice_free(Lattice* L) { delete L; }
size_t lattice_bytes(const Lattice*) { return 0; }
}  // namespace gahhg
