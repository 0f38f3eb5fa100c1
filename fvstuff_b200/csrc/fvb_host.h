// fvb_host.h -- host-side helpers shared by the C-ABI implementation files.
#pragma once
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "fvb_aux.h"

namespace fvb {

// Sizes of one grid's internal buffers.
struct Geometry {
    int n, g, np;
    int pitch, xoff;
    long long plane;
    size_t elem;   // bytes per state word
    int nbuf;      // padded 4-variable buffers (3: state + 2 stage outputs; 6 for F32C)
    size_t bytes;  // all buffers
};

// A named range on a profiler's timeline (Nsight Systems / Compute) around a
// host entry point; without a profiler attached it costs next to nothing.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

fvb_status fail(fvb_status st, const char *fmt, ...);
fvb_status cuda_fail(cudaError_t e, const char *what);
int prec_internal(int prec);
size_t prec_elem(int prec);
Geometry make_geometry(int n, int g, int prec);
void grid_pointers(GridDev &gd, void *base, const Geometry &G, int prec);
BufView view_of(const GridDev &gd);
void tile_dims(int shape, int n, int &tiles_x, int &tiles);
void case_defaults(fvb_case *c, int kind, double x0, double y0, double L);

// tile variant for a grid size (fvb_tune.cpp)
int autotune_shape(int prec, int order, int n);

// KEEP flux family (fvb_keep.cu): tiles of a grid, one stage (entropy-
// distance pass + fused stage kernel), and the wave-speed max of a state
void keep_tiles(int n, int &tiles_x, int &tiles);
cudaError_t keep_launch_stage(const GridDev &gd, int stage, int tiles, cudaStream_t s);
cudaError_t keep_lam_into(const GridDev &gd, cudaStream_t s);

// rec3 + HLLC + 2x2-block Zhang-Shu (fvb_rec3.cu): tiles, one fused stage,
// the limiter pass over a whole state, max wave speed, fv_rec3's initial
// states (0 Sod, 1 paper vortex, 2 Gresho with background pressure p0)
void rec3_tiles(int n, int &tiles_x, int &tiles);
cudaError_t rec3_launch_stage(const GridDev &gd, int stage, int tiles, cudaStream_t s);
cudaError_t rec3_limit_into(const GridDev &gd, void *buf, cudaStream_t s);
cudaError_t rec3_lam_into(const GridDev &gd, cudaStream_t s);
cudaError_t rec3_init_case(const GridDev &gd, int icase, double p0, cudaStream_t s);

// UP + HLLC + Ducros-gated D2 viscosity of fv_up7_ducros_2d.cu.bak
// (fvb_d2av.cu): ghost width of an order (the sensor reaches 3 cells), tiles,
// one fused stage, the wave-speed max of a state, and the Ducros weight of
// every cell as FP32 (frames)
int d2av_ghost(int order);
void d2av_tiles(int n, int &tiles_x, int &tiles);
cudaError_t d2av_launch_stage(const GridDev &gd, int order, int stage, int tiles, const D2Params &av,
                              cudaStream_t s);
cudaError_t d2av_lam_into(const GridDev &gd, cudaStream_t s);
cudaError_t d2av_sensor_into(const GridDev &gd, double sc, float *out, cudaStream_t s);

}  // namespace fvb
