// fvb_host.h -- host-side helpers shared by the C-ABI implementation files.
#pragma once
#include <string>

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

// KEEP flux family (fvb_keep.cpp), reached through the same fvb_solver handle
fvb_status keep_create(const fvb_config *cfg, fvb_solver **out);
void keep_destroy(fvb_solver *s);
fvb_status keep_init_case(fvb_solver *s, const fvb_case *c);
fvb_status keep_set_state(fvb_solver *s, const void *src, int layout, int dtype, int where, int interior_only);
fvb_status keep_get_state(fvb_solver *s, void *dst, int layout, int dtype, int where, int interior_only);
fvb_status keep_step(fvb_solver *s, int nsteps, double t_stop);
fvb_status keep_sync(fvb_solver *s, fvb_stats *st);
fvb_status keep_stats_sums(fvb_solver *s, fvb_stats *st);

}  // namespace fvb
