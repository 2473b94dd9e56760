/*
 * refshim.h - force-included header that lets the reference's CUDA sources
 * (source/GPISPAHHG.cu, GPISPPolygon.cu, GPISPTP.cu, GPISP.cu) compile and run
 * as host C++.  TEST INFRASTRUCTURE ONLY: the product never links this.
 *
 * What it maps:
 *   __global__/__device__  -> plain functions;
 *   threadIdx/blockIdx/blockDim -> thread-local values set by the launcher;
 *   kernel<<<b, t>>>(args)  -> REFSHIM_LAUNCH(kernel, b, t)(args) (the build
 *                              recipe rewrites the launch syntax), which runs
 *                              every (block, thread) either serially in tid
 *                              order (parity mode) or with OpenMP (timing);
 *   atomicAdd               -> __atomic_fetch_add;
 *   cudaMalloc/Free/Memcpy/Memset -> host memory (cudaMalloc zero-fills; a
 *                              second cudaFree of a pointer is ignored, because
 *                              GAHHG::clear frees dev_r[0] three times,
 *                              source/GPISPAHHG.cu:1937-1942);
 *   sin/cos                 -> the canonical sine/cosine of gahhg_canon.h, so
 *                              the reference's LL2XYZ/FakeLL2XYZ produce the
 *                              same XYZ bits as the GPU path.
 */
#ifndef GAHHG_REFSHIM_H
#define GAHHG_REFSHIM_H

/* Every standard header the reference pulls in, before the macros below. */
#include <cmath>
#include <math.h>
#include <cfloat>
#include <float.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <fcntl.h>

#include "gahhg_canon.h"

#define __global__
#define __device__
#define __host__

struct refshim_dim3 { unsigned int x, y, z; };
extern thread_local refshim_dim3 threadIdx;
extern thread_local refshim_dim3 blockIdx;
extern thread_local refshim_dim3 blockDim;

static inline int atomicAdd(int* p, int v) { return __atomic_fetch_add(p, v, __ATOMIC_RELAXED); }

/* ---- CUDA runtime stand-ins (host memory) ---- */
typedef int cudaError_t;
enum cudaMemcpyKind {
    cudaMemcpyHostToHost = 0,
    cudaMemcpyHostToDevice = 1,
    cudaMemcpyDeviceToHost = 2,
    cudaMemcpyDeviceToDevice = 3
};
cudaError_t refshim_malloc(void** p, size_t n);
cudaError_t cudaFree(void* p);
template <class T> static inline cudaError_t cudaMalloc(T** p, size_t n)
{
    return refshim_malloc((void**)p, n);
}
static inline cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind)
{
    if (n) memmove(d, s, n);
    return 0;
}
static inline cudaError_t cudaMemset(void* d, int v, size_t n)
{
    if (n) memset(d, v, n);
    return 0;
}
static inline cudaError_t cudaDeviceSynchronize() { return 0; }

/* The vendored scan (source/scan/scan.cu:104-112) is an exclusive prefix sum. */
void myscan(int* dev_output, int* dev_input, int length, bool bcao);

/* ---- kernel launcher ---- */
namespace refshim {
extern int g_threads;     /* <= 1: serial in tid order; > 1: OpenMP threads */
extern int g_reverse;     /* serial mode only: run tids in descending order */
void set_index(long long tid, unsigned nt);
template <class K> struct Launch {
    K k;
    unsigned nb, nt;
    template <class... A> void operator()(A... a) const
    {
        long long total = (long long)nb * (long long)nt;
        if (g_threads <= 1) {
            for (long long i = 0; i < total; i++) {
                long long t = g_reverse ? total - 1 - i : i;
                set_index(t, nt);
                k(a...);
            }
        } else {
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 256)
            for (long long t = 0; t < total; t++) {
                set_index(t, nt);
                k(a...);
            }
        }
    }
};
template <class K> static inline Launch<K> launch(K k, unsigned nb, unsigned nt)
{
    return Launch<K>{k, nb, nt};
}
} // namespace refshim

#define REFSHIM_LAUNCH(kern, nb, nt) ::refshim::launch(kern, (unsigned)(nb), (unsigned)(nt))

/* ---- canonical conversion for the reference's LL2XYZ / FakeLL2XYZ ---- */
static inline double refshim_sin(double x)
{
    double s, c;
    gahhg_canon_sincos(x, &s, &c);
    return s;
}
static inline double refshim_cos(double x)
{
    double s, c;
    gahhg_canon_sincos(x, &s, &c);
    return c;
}
#define sin(x) refshim_sin(x)
#define cos(x) refshim_cos(x)

#endif
