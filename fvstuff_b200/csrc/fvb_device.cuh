// fvb_device.cuh -- device helpers shared by the stage kernels of both flux
// families: precision traits, padded addressing, stores with ghost images,
// the compensated FP32 add and the device-side step control.
#pragma once
#include "fvb_internal.h"
#include "fvb_physics.cuh"

namespace fvb {

template <int PREC> struct PrecT;
template <> struct PrecT<P64> { using R = double; using RR = double; };
template <> struct PrecT<P32> { using R = float; using RR = double; };
template <> struct PrecT<P32C> { using R = float; using RR = float; };

__device__ __forceinline__ long long gidx(const GridDev &gd, int q, int j, int i)
{
    // interior coordinates (j, i), negative or >= n inside the ghost ring
    return (long long)q * gd.plane + (long long)(j + gd.g) * gd.pitch + (i + gd.g) + gd.xoff;
}

// Ghost images of cell i along one axis (index 0 is the cell itself).
//   reflect:      i < g -> -1-i,  i >= n-g -> 2n-1-i  (normal momentum negated)
//   periodic:     i < g -> i+n,   i >= n-g -> i-n
//   transmissive: i == 0 -> -1..-g,  i == n-1 -> n..n+g-1
// (the ghost fills of fv_up7_ducros_2d.cu:338-362 and keep_fv_euler_2d.cu:
// 224-243, and zero-gradient, seen from the cell side).  Computed
// arithmetically, so no per-thread arrays are needed.
__device__ __forceinline__ int n_images(int i, int n, int g, int bc)
{
    if (bc == FVB_BC_REFLECT || bc == FVB_BC_PERIODIC) return 1 + (i < g) + (i >= n - g);
    return 1 + (i == 0 ? g : 0) + (i == n - 1 ? g : 0);
}

__device__ __forceinline__ int image_of(int k, int i, int n, int g, int bc, bool &flip)
{
    flip = false;
    if (k == 0) return i;
    const bool low = (k == 1 && i < g);
    if (bc == FVB_BC_REFLECT) {
        flip = true;
        return low ? -1 - i : 2 * n - 1 - i;
    }
    if (bc == FVB_BC_PERIODIC) return low ? i + n : i - n;
    if (i == 0 && k <= g) return -k;
    return n - 1 + (i == 0 ? k - g : k);
}

// Store a cell value into the interior and all its ghost images.
template <class R>
__device__ __forceinline__ void put_cell(const GridDev &gd, R *buf, int j, int i, const R v[4])
{
    const long long pl = gd.plane;
    const long long c = gidx(gd, 0, j, i);
    buf[c] = v[0];
    buf[c + pl] = v[1];
    buf[c + 2 * pl] = v[2];
    buf[c + 3 * pl] = v[3];
    const int g = gd.g, n = gd.n;
    if (i >= g && i < n - g && j >= g && j < n - g) return;
    const int nx = n_images(i, n, g, gd.bcx), ny = n_images(j, n, g, gd.bcy);
    for (int ka = 0; ka < ny; ++ka) {
        bool fy;
        const int y = image_of(ka, j, n, g, gd.bcy, fy);
        for (int kb = (ka == 0 ? 1 : 0); kb < nx; ++kb) {
            bool fx;
            const int x = image_of(kb, i, n, g, gd.bcx, fx);
            const long long e = gidx(gd, 0, y, x);
            buf[e] = v[0];
            buf[e + pl] = fx ? -v[1] : v[1];
            buf[e + 2 * pl] = fy ? -v[2] : v[2];
            buf[e + 3 * pl] = v[3];
        }
    }
}

// Store two cell values that share a layout (the hi and lo words of the
// compensated state) into the interior and all their ghost images.
template <class R>
__device__ __forceinline__ void put_cell2(const GridDev &gd, R *bufA, R *bufB, int j, int i, const R va[4],
                                          const R vb[4])
{
    const long long pl = gd.plane;
    const long long c = gidx(gd, 0, j, i);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        bufA[c + q * pl] = va[q];
        bufB[c + q * pl] = vb[q];
    }
    const int g = gd.g, n = gd.n;
    if (i >= g && i < n - g && j >= g && j < n - g) return;
    const int nx = n_images(i, n, g, gd.bcx), ny = n_images(j, n, g, gd.bcy);
    for (int ka = 0; ka < ny; ++ka) {
        bool fy;
        const int y = image_of(ka, j, n, g, gd.bcy, fy);
        for (int kb = (ka == 0 ? 1 : 0); kb < nx; ++kb) {
            bool fx;
            const int x = image_of(kb, i, n, g, gd.bcx, fx);
            const long long e = gidx(gd, 0, y, x);
            bufA[e] = va[0]; bufB[e] = vb[0];
            bufA[e + pl] = fx ? -va[1] : va[1]; bufB[e + pl] = fx ? -vb[1] : vb[1];
            bufA[e + 2 * pl] = fy ? -va[2] : va[2]; bufB[e + 2 * pl] = fy ? -vb[2] : vb[2];
            bufA[e + 3 * pl] = va[3]; bufB[e + 3 * pl] = vb[3];
        }
    }
}

// Error-free sum of a double-float (hi, lo) and a float increment d
// (Knuth TwoSum for hi + d, then Dekker FastTwoSum to renormalise).
__device__ __forceinline__ void df_add(float &hi, float &lo, float d)
{
    float s = __fadd_rn(hi, d);
    float bb = __fsub_rn(s, hi);
    float err = __fadd_rn(__fsub_rn(hi, __fsub_rn(s, bb)), __fsub_rn(d, bb));
    float l = __fadd_rn(lo, err);
    float h2 = __fadd_rn(s, l);
    lo = __fsub_rn(l, __fsub_rn(h2, s));
    hi = h2;
}

// does any grid of this launch load through TMA (a single-grid launch
// decides by its descriptor; batched grids all carry descriptors)
__device__ __forceinline__ bool gd_has_tma(const StageArgs &a)
{
    return a.grids != nullptr || a.grid.tmap != nullptr;
}

// Step control of one grid for one stage, evaluated from `s`, a copy of the
// grid's Ctrl taken during this stage (or the Ctrl itself), with the
// control writes going to `c`.  `leader` (one thread of the launch per grid:
// thread 0 of CTA 0 of a single-grid launch, the thread that publishes the
// header of the grid's tile 0 in a batched launch, thread 0 of the tile-0
// CTA of the KEEP and rec3 kernels) also writes the stage's control updates:
// dt, `active` and `clamped` in stage 1, the wave-speed accumulator reset in
// stage 2.  Every other caller only reads.  The fields a stage reads are
// never written during it, except `status` in stage 1, which the leader may
// set to a stop that every reader derives for itself from the same inputs.
template <int PREC>
__device__ TileCtl step_control(const Ctrl &s, Ctrl *c, int stage, bool leader)
{
    TileCtl k{0.0, 0, 0};
    if (stage == 0) { k.run = 1; return k; }
    if (stage == 1) {
        double t = s.t, ts = s.t_stop;
        // the FP32 form keeps float time, as the shipped solver does: a stop
        // time is reached when the float time reaches its float value
        const bool reached = PREC == P32 ? !((float)t < (float)ts) : !(t < ts);
        if (s.status != 0 || reached) {
            if (leader) c->active = 0;
            return k;
        }
        double lam = __longlong_as_double((long long)s.lam_acc);
        if (!(lam > 0.0)) {
            if (leader) { c->status = FVB_ERR_BLOWUP; c->active = 0; }
            return k;
        }
        double dt;
        int clamped = 0;
        if (PREC == P64) {
            dt = s.cfl * s.h / lam;
            if (t + dt > ts) { dt = ts - t; clamped = 1; }
            if (dt < 1e-14) {
                if (leader) { c->status = FVB_ERR_DT_UNDERFLOW; c->active = 0; }
                return k;
            }
        } else if (PREC == P32) {
            // float time and dt, as the shipped solver keeps them
            float tf = (float)t, tsf = (float)ts;
            float d = (float)s.cfl * (float)s.h / (float)lam;
            if (tf + d > tsf) { d = tsf - tf; clamped = 1; }
            if (d < 1e-14f) {
                if (leader) { c->status = FVB_ERR_DT_UNDERFLOW; c->active = 0; }
                return k;
            }
            dt = d;
        } else {
            // FP32 dt, FP64 accumulated time landing exactly on t_stop
            float d = (float)(s.cfl * s.h) / (float)lam;
            if (t + (double)d > ts) { d = (float)(ts - t); clamped = 1; }
            if (d < 1e-14f) {
                if (leader) { c->status = FVB_ERR_DT_UNDERFLOW; c->active = 0; }
                return k;
            }
            dt = d;
        }
        if (leader) {
            c->dt = dt;
            c->active = 1;
            c->clamped = clamped;
            c->lam_cur = s.lam_acc;
        }
        k.dt = dt;
        k.run = 1;
        return k;
    }
    if (!s.active) {
        k.copy = (stage == 3 && PREC == P32C);
        return k;
    }
    k.dt = s.dt;
    k.run = 1;
    if (stage == 2 && leader) c->lam_acc = 0ull;
    return k;
}

template <int PREC>
__device__ __forceinline__ TileCtl tile_control(Ctrl *c, int stage, bool leader)
{
    return step_control<PREC>(*c, c, stage, leader);
}

// end of stage 3 (leader): time and step count advance
template <int PREC>
__device__ __forceinline__ void leader_finish_from(const Ctrl &s, Ctrl *c)
{
    double t = s.t, dt = s.dt;
    if (PREC == P32) t = (double)((float)t + (float)dt);
    else if (PREC == P32C) t = s.clamped ? s.t_stop : t + dt;
    else t = t + dt;
    c->t = t;
    c->step = s.step + 1;
}

template <int PREC>
__device__ __forceinline__ void leader_finish(Ctrl *c)
{
    leader_finish_from<PREC>(*c, c);
}

}  // namespace fvb
