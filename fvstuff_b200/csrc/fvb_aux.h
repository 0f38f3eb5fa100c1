// fvb_aux.h -- declarations of the kernels in fvb_aux.cu.
#pragma once
#include "fvb_internal.h"

namespace fvb {

// geometry of an internal padded buffer (see GridDev)
struct BufView {
    int n, g;
    int pitch, xoff;
    long long plane;
};

// geometry of a caller array: IDX_P padded (np = n + 2g) or interior (n x n)
struct ExtView {
    int interior;
    int g, np;
    int layout;  // fvb_layout
    int dtype;   // fvb_dtype
};

// coefficients of the D2 artificial viscosity of the .bak scheme
// (fv_up7_ducros_2d.cu.bak:742-745): Ducros-gated C2, global Cg, sensor
// sound-speed scale sc
struct D2Params {
    double c2, cg, sc;
};

// internal state kinds
enum { INT_PRIM64 = 0, INT_PRIM32 = 1, INT_CONS_HILO = 2, INT_CONS64 = 3 };

template <class R>
cudaError_t bc_fill(R *buf, const BufView &v, int bcx, int bcy, cudaStream_t s);
// circular Sod evaluated in FP32 as the shipped FP32 solver does (the FP32 form's initial state)
cudaError_t init_sod_prim32(float *out, int n, double x0, double y0, double length, const fvb_case &c,
                            cudaStream_t s);
cudaError_t init_case_prim64(double *out, int n, double x0, double y0, double h, double gam, const fvb_case &c,
                             cudaStream_t s);
cudaError_t import_state(const void *src, const ExtView &e, void *dst, void *dst_lo, const BufView &v,
                         int internal, double gam, cudaStream_t s);
cudaError_t export_state(const void *src, const void *src_lo, const BufView &v, int internal, void *dst,
                         const ExtView &e, double gam, cudaStream_t s);
cudaError_t lam_into(const void *st, const BufView &v, int internal, double gam, unsigned long long *acc,
                     cudaStream_t s);
cudaError_t sums_partials(const void *st, const void *lo, const BufView &v, int internal, double gam,
                          double *part, int blocks, cudaStream_t s);
template <class R>
cudaError_t rk3_stage_ref(int stage, R *Uo, const R *U0, const R *Uk, const R *L, R dt, int n, int np, int g,
                          double gam, cudaStream_t s);
cudaError_t max_ref(const void *x, size_t n, void *out, int dtype, cudaStream_t s);
cudaError_t ctrl_set(Ctrl *c, double t_stop, int reset, double t0, double cfl, double h, cudaStream_t s);
// rho, vorticity, Ducros cell sensor, |v|, p (5 x n x n floats) from an FP32
// primitive IDX_P array with its ghost ring
cudaError_t frame_fields(const float *prim, int n, int g, int np, double h, float *out, cudaStream_t s);

}  // namespace fvb
