// geom.cuh - grid record types and FP64 vector arithmetic shared by the host
// and the device code of the GAHHG path.
//
// Grid records keep the reference's field layout (source/common.h:169-186,
// source/GPISPAHHG.cuh:12-20): the storage figures in report.txt are computed
// from these sizes (48 B per border, 28 B per cell, 24 B per vertex), and the
// tests compare whole grid arrays against the reference built for the CPU.
//
// D3 arithmetic evaluates every expression in the same order as the
// reference's devdouble3 (source/GPISPDS.cuh:12-107): a+b, a-b, a*k,
// a/k = a*(1.0/k), normalize = a*(1.0/sqrt(x*x+y*y+z*z)), cross, dot.  All
// CUDA sources are compiled with --fmad=false and the host with
// -ffp-contract=off, so each operation is one IEEE-754 rounding on both sides
// and the grids come out bit-identical.
#pragma once

#include <math.h>
#include <stdint.h>

#ifdef __CUDACC__
#define GHD __host__ __device__ __forceinline__
#else
#define GHD inline
#endif

namespace gahhg {

// Cell types (source/GPISPParam.h:9-11).
enum { CELL_UNDEFINED = 0, CELL_OUT = 1, CELL_IN = 2 };
// Edge/border intersection codes (source/GPISPParam.h:13-17).
enum { INTER_NO = 0, INTER_X = 1, INTER_T1 = 2, INTER_T2 = 3, INTER_OVERLAP = 4 };

constexpr double TRAVEL_EPSILON = 1.0e-5;    // source/GPISPParam.h:6
constexpr double POSITION_EPSILON = 1.0e-8;  // source/GPISPParam.h:7

struct Border {      // half-edge of a cell; AHHGBorder (source/common.h:169-176)
    int parent;      // owning cell
    int partner;     // twin half-edge in the neighbouring cell, -1 if none
    int v[2];        // vertex indices, counter-clockwise seen from outside
    int subcell;     // border subcell created on this border, -1 if none
    int id;          // position in the owning cell's ring
    double n[3];     // inward normal: normalize(v0 x (v1 - v0))
};
static_assert(sizeof(Border) == 48, "Border must stay 48 bytes");

struct Cell {        // AHHGCell (source/common.h:178-186)
    int bstart, bnum;
    int rstart, rnum;    // edge refs (bottom level); rnum 999 marks a crossed cell
    int upcell, subcell;
    int type;
};
static_assert(sizeof(Cell) == 28, "Cell must stay 28 bytes");

struct Level {       // GAHHGGrid (source/GPISPAHHG.cuh:12-20)
    int vstart, vnum, bstart, bnum, cstart, cnum, rnum;
};

struct D3 {
    double x, y, z;
};

GHD D3 d3(double x, double y, double z) { return D3{x, y, z}; }
GHD D3 operator+(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
GHD D3 operator-(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
GHD D3 operator-(D3 a) { return D3{-a.x, -a.y, -a.z}; }
GHD D3 operator*(D3 a, double k) { return D3{a.x * k, a.y * k, a.z * k}; }
GHD D3 operator/(D3 a, double k)
{
    double s = 1.0 / k;
    return D3{a.x * s, a.y * s, a.z * s};
}
GHD double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
GHD double squarelen(D3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
GHD D3 cross(D3 a, D3 b)
{
    return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
GHD D3 normalize(D3 a)
{
    double t = 1.0 / sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
    return D3{a.x * t, a.y * t, a.z * t};
}
// device_getENormal (source/GPISPAHHG.cu:18-25)
GHD D3 edge_normal(D3 v0, D3 v1) { return normalize(cross(v0, v1 - v0)); }

GHD bool less_zero(double a) { return a < -POSITION_EPSILON; }
GHD bool gre_zero(double a) { return a > POSITION_EPSILON; }
GHD bool equ_zero(double a) { return a < POSITION_EPSILON && a > -POSITION_EPSILON; }
GHD bool less_equ_zero(double a) { return a < POSITION_EPSILON; }
GHD bool gre_equ_zero(double a) { return a > -POSITION_EPSILON; }

}  // namespace gahhg
