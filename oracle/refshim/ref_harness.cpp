// ref_harness.cpp - C API over the reference's own GAHHG code compiled for the
// CPU (TEST INFRASTRUCTURE; used by tests/ and by bench.py's reference arm).
//
// The calls mirror the reference driver (source/GPISP.cu:15-70):
//   loadPolyFromTXT -> createAHHGInit -> createAHHG(maxdepth) -> classifyAHHG
//   -> test() -> getStat(),
// except that query points come from a lon/lat array instead of a CSV file;
// they are converted exactly as loadTPFromCSV does (source/GPISPTP.cu:64-69,
// FakeLLVertex::FakeLL2XYZ).
#include "refshim.h"
#include "GPISPAHHG.cuh"

#include <vector>

extern "C" {

struct ref_stats {
    int gnum;
    int pv_num;
    int vnum, bnum, cnum, rnum;
    int cpu_space;
    int gpu_min_space;
    float gamma;
    double create_s, classify_s, query_s;
    int in_count;
};

void ref_set_threads(int n, int reverse)
{
    refshim::g_threads = n;
    refshim::g_reverse = reverse;
}

// Returns NULL when the polygon file fails to load (the loader prints why).
void* ref_open(const char* polyfile, int maxdepth, int autodepth)
{
    GPISP* g = new GPISP();
    g->pParam = new GPISPParam();
    g->pParam->autoDepth = autodepth != 0;
    if (maxdepth > 0) g->pParam->maxDepth = maxdepth;
    strncpy(g->pParam->polyFileName, polyfile, sizeof(g->pParam->polyFileName) - 1);
    g->pPolygon = new GPISPPolygon;
    if (g->pPolygon->loadPolyFromTXT(g->pParam->polyFileName) == -1) {
        delete g;
        return nullptr;
    }
    g->pStat = new GPISPStat;
    g->pAHHG = new GAHHG(g->pPolygon, g->pParam, g->pStat);
    g->createAHHGInit();
    g->createAHHG(g->pParam->maxDepth);
    g->classifyAHHG();
    return g;
}

// labels_out: one int per point, the reference's dev_result values
// (0 = never written / undefined, 1 = OUT, 2 = IN).
void ref_query(void* h, const double* lonlat, int n, int* labels_out)
{
    GPISP* g = (GPISP*)h;
    if (g->pTP) delete g->pTP;
    GPISPTP* tp = new GPISPTP;
    tp->tpNum = n;
    tp->tpll = new LLVertex[n];
    tp->tp = new mydouble3[n];
    tp->result = new int[n];
    for (int i = 0; i < n; i++) {
        tp->tpll[i].lo = lonlat[2 * i];
        tp->tpll[i].la = lonlat[2 * i + 1];
        FakeLLVertex f(tp->tpll[i]);
        tp->tp[i] = f.FakeLL2XYZ();
    }
    cudaMalloc((void**)&tp->dev_tp, sizeof(devdouble3) * n);
    cudaMemcpy(tp->dev_tp, tp->tp, sizeof(devdouble3) * n, cudaMemcpyHostToDevice);
    cudaMalloc((void**)&tp->dev_result, sizeof(int) * n);
    g->pTP = tp;
    g->test();
    memcpy(labels_out, tp->result, sizeof(int) * n);
}

void ref_stats_get(void* h, ref_stats* s)
{
    GPISP* g = (GPISP*)h;
    if (g->pTP) g->getStat();
    GAHHG* a = g->pAHHG;
    const GAHHGGrid& last = a->g[a->gnum - 1];
    s->gnum = a->gnum;
    s->pv_num = g->pPolygon->pv_num;
    s->vnum = last.vstart + last.vnum;
    s->bnum = last.bstart + last.bnum;
    s->cnum = last.cstart + last.cnum;
    s->rnum = last.rnum;
    s->cpu_space = (int)(sizeof(GAHHG) + sizeof(GAHHGGrid) * a->gnum + sizeof(GPISPParam) + sizeof(GPISPStat));
    s->gpu_min_space = (int)(sizeof(devdouble3) * s->vnum + sizeof(AHHGBorder) * s->bnum +
                             sizeof(AHHGCell) * s->cnum + sizeof(int) * s->rnum);
    s->gamma = g->pStat->gamma;
    s->create_s = g->pStat->createAHHGTime;
    s->classify_s = g->pStat->classifyAHHGTime;
    s->query_s = g->pStat->PISPTime;
    s->in_count = g->pStat->inTpNum;
}

// Copies the grid arrays: levels (7 ints each), vertices (3 doubles),
// borders (AHHGBorder, 48 B), cells (AHHGCell, 28 B), refs (ints).
// Any output pointer may be NULL.
void ref_grid_export(void* h, int* levels, double* v, void* b, void* c, int* refs)
{
    GPISP* g = (GPISP*)h;
    GAHHG* a = g->pAHHG;
    const GAHHGGrid& last = a->g[a->gnum - 1];
    if (levels) memcpy(levels, a->g, sizeof(GAHHGGrid) * a->gnum);
    if (v) memcpy(v, a->dev_v, sizeof(devdouble3) * (last.vstart + last.vnum));
    if (b) memcpy(b, a->dev_b, sizeof(AHHGBorder) * (last.bstart + last.bnum));
    if (c) memcpy(c, a->dev_c, sizeof(AHHGCell) * (last.cstart + last.cnum));
    if (refs) memcpy(refs, a->dev_r[0], sizeof(int) * last.rnum);
}

// The loaded polygon: canonical vertex XYZ (3 doubles each) and edge list.
void ref_polygon_export(void* h, double* pv, int* pe)
{
    GPISP* g = (GPISP*)h;
    if (pv) memcpy(pv, g->pPolygon->pv, sizeof(mydouble3) * g->pPolygon->pv_num);
    if (pe) memcpy(pe, g->pPolygon->pe, sizeof(int) * 2 * g->pPolygon->pv_num);
}

void ref_close(void* h)
{
    GPISP* g = (GPISP*)h;
    delete g;
}

// The level-0 grid this build supplies for the closed initgrid0.
void ref_grid0_export(double* v, void* b, void* c)
{
    myArray<mydouble3> vv(160);
    myArray<AHHGBorder> bb(480);
    myArray<AHHGCell> cc(84);
    initgrid0(&vv, &bb, &cc);
    memcpy(v, vv.elem, sizeof(mydouble3) * vv.curNum);
    memcpy(b, bb.elem, sizeof(AHHGBorder) * bb.curNum);
    memcpy(c, cc.elem, sizeof(AHHGCell) * cc.curNum);
}

int ref_sizeof(int which)
{
    switch (which) {
    case 0: return (int)sizeof(AHHGBorder);
    case 1: return (int)sizeof(AHHGCell);
    case 2: return (int)sizeof(GAHHGGrid);
    case 3: return (int)(sizeof(GAHHG) + sizeof(GPISPParam) + sizeof(GPISPStat));
    default: return -1;
    }
}

}  // extern "C"
