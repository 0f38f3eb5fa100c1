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

// Coordinates of cell i and of every ghost cell that mirrors it along one
// axis; flip marks reflected images (normal momentum negated).
__device__ __forceinline__ int mirror_images(int i, int n, int g, int bc, int *pos, bool *flip)
{
    int k = 0;
    pos[k] = i; flip[k++] = false;
    if (bc == FVB_BC_REFLECT) {
        if (i < g) { pos[k] = -1 - i; flip[k++] = true; }
        if (i >= n - g) { pos[k] = 2 * n - 1 - i; flip[k++] = true; }
    } else if (bc == FVB_BC_PERIODIC) {
        if (i < g) { pos[k] = i + n; flip[k++] = false; }
        if (i >= n - g) { pos[k] = i - n; flip[k++] = false; }
    } else {
        if (i == 0) for (int m = 1; m <= g; ++m) { pos[k] = -m; flip[k++] = false; }
        if (i == n - 1) for (int m = 0; m < g; ++m) { pos[k] = n + m; flip[k++] = false; }
    }
    return k;
}

// Store a cell value into the interior and all its ghost images.
template <class R>
__device__ __forceinline__ void put_cell(const GridDev &gd, R *buf, int j, int i, const R v[4])
{
    long long c = gidx(gd, 0, j, i);
    buf[c] = v[0];
    buf[c + gd.plane] = v[1];
    buf[c + 2 * gd.plane] = v[2];
    buf[c + 3 * gd.plane] = v[3];
    const int g = gd.g, n = gd.n;
    if (i >= g && i < n - g && j >= g && j < n - g) return;
    int xs[12], ys[12];
    bool fx[12], fy[12];
    int nx = mirror_images(i, n, g, gd.bcx, xs, fx);
    int ny = mirror_images(j, n, g, gd.bcy, ys, fy);
    for (int a = 0; a < ny; ++a)
        for (int b = 0; b < nx; ++b) {
            if (a == 0 && b == 0) continue;
            long long e = gidx(gd, 0, ys[a], xs[b]);
            buf[e] = v[0];
            buf[e + gd.plane] = fx[b] ? -v[1] : v[1];
            buf[e + 2 * gd.plane] = fy[a] ? -v[2] : v[2];
            buf[e + 3 * gd.plane] = v[3];
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

// Step control, evaluated by thread 0 of each CTA for its tile's grid.
template <int PREC>
__device__ TileCtl tile_control(Ctrl *c, int stage, bool leader)
{
    TileCtl s{0.0, 0, 0};
    if (stage == 0) { s.run = 1; return s; }
    if (stage == 1) {
        double t = c->t, ts = c->t_stop;
        if (c->status != 0 || !(t < ts)) {
            if (leader) c->active = 0;
            return s;
        }
        double lam = __longlong_as_double((long long)c->lam_acc);
        if (!(lam > 0.0)) {
            if (leader) { c->status = FVB_ERR_BLOWUP; c->active = 0; }
            return s;
        }
        double dt;
        int clamped = 0;
        if (PREC == P64) {
            dt = c->cfl * c->h / lam;
            if (t + dt > ts) { dt = ts - t; clamped = 1; }
            if (dt < 1e-14) {
                if (leader) { c->status = FVB_ERR_DT_UNDERFLOW; c->active = 0; }
                return s;
            }
        } else if (PREC == P32) {
            // float time and dt, as the shipped solver keeps them
            float tf = (float)t, tsf = (float)ts;
            float d = (float)c->cfl * (float)c->h / (float)lam;
            if (tf + d > tsf) { d = tsf - tf; clamped = 1; }
            if (d < 1e-14f) {
                if (leader) { c->status = FVB_ERR_DT_UNDERFLOW; c->active = 0; }
                return s;
            }
            dt = d;
        } else {
            // FP32 dt, FP64 accumulated time landing exactly on t_stop
            float d = (float)(c->cfl * c->h) / (float)lam;
            if (t + (double)d > ts) { d = (float)(ts - t); clamped = 1; }
            if (d < 1e-14f) {
                if (leader) { c->status = FVB_ERR_DT_UNDERFLOW; c->active = 0; }
                return s;
            }
            dt = d;
        }
        if (leader) {
            c->dt = dt;
            c->active = 1;
            c->clamped = clamped;
            c->lam_cur = c->lam_acc;
        }
        s.dt = dt;
        s.run = 1;
        return s;
    }
    if (!c->active) {
        s.copy = (stage == 3 && PREC == P32C);
        return s;
    }
    s.dt = c->dt;
    s.run = 1;
    if (stage == 2 && leader) c->lam_acc = 0ull;
    return s;
}

template <int PREC>
__device__ __forceinline__ void leader_finish(Ctrl *c)
{
    double t = c->t, dt = c->dt;
    if (PREC == P32) t = (double)((float)t + (float)dt);
    else if (PREC == P32C) t = c->clamped ? c->t_stop : t + dt;
    else t = t + dt;
    c->t = t;
    c->step = c->step + 1;
}

}  // namespace fvb
