// refshim.cpp - runtime half of refshim.h (test infrastructure only).
#include "refshim.h"

#include <mutex>
#include <unordered_set>

thread_local refshim_dim3 threadIdx;
thread_local refshim_dim3 blockIdx;
thread_local refshim_dim3 blockDim;

namespace refshim {
int g_threads = 1;
int g_reverse = 0;

void set_index(long long tid, unsigned nt)
{
    threadIdx.x = (unsigned)(tid % nt);
    threadIdx.y = threadIdx.z = 0;
    blockIdx.x = (unsigned)(tid / nt);
    blockIdx.y = blockIdx.z = 0;
    blockDim.x = nt;
    blockDim.y = blockDim.z = 1;
}

static std::mutex g_mu;
static std::unordered_set<void*>& live()
{
    static std::unordered_set<void*> s;
    return s;
}
} // namespace refshim

cudaError_t refshim_malloc(void** p, size_t n)
{
    void* q = calloc(n ? n : 1, 1);
    *p = q;
    if (!q) return 2;
    std::lock_guard<std::mutex> g(refshim::g_mu);
    refshim::live().insert(q);
    return 0;
}

cudaError_t cudaFree(void* p)
{
    if (!p) return 0;
    {
        std::lock_guard<std::mutex> g(refshim::g_mu);
        auto it = refshim::live().find(p);
        if (it == refshim::live().end()) return 0;  // repeated free: ignored
        refshim::live().erase(it);
    }
    free(p);
    return 0;
}

void myscan(int* out, int* in, int length, bool)
{
    int acc = 0;
    for (int i = 0; i < length; i++) {
        int v = in[i];
        out[i] = acc;
        acc += v;
    }
}
