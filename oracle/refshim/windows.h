/* Stand-in for <windows.h> so the reference sources build on Linux.
 * Provides only what source/GPISPParam.h and the loaders use. */
#pragma once
#include <time.h>
#include <stdio.h>
#include <string.h>
typedef long long __int64;
typedef union { struct { unsigned int LowPart; int HighPart; } u; long long QuadPart; } LARGE_INTEGER;
static inline int QueryPerformanceFrequency(LARGE_INTEGER* f) { f->QuadPart = 1000000000LL; return 1; }
static inline int QueryPerformanceCounter(LARGE_INTEGER* c)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    c->QuadPart = (long long)ts.tv_sec * 1000000000LL + ts.tv_nsec;
    return 1;
}
#define sscanf_s sscanf
template <size_t N> static inline int strcpy_s(char (&d)[N], const char* s)
{
    strncpy(d, s, N - 1);
    d[N - 1] = 0;
    return 0;
}
static inline int fopen_s(FILE** f, const char* name, const char* mode)
{
    *f = fopen(name, mode);
    return *f ? 0 : 1;
}
static inline int localtime_s(struct tm* t, const time_t* tt) { return localtime_r(tt, t) ? 0 : 1; }
