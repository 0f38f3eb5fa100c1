// fvb_stage.cu -- the fused SSP-RK3 stage kernel.
//
// One launch = one RK stage of one grid (or of every grid of a batch, through
// a tile table).  Per tile of TX x TY interior cells a CTA
//   1. stages the (TX+2g) x (TY+2g) halo tile of the stage-input state into
//      shared memory as primitives,
//   2. evaluates every face of the tile once: UP-ORDER reconstruction of the
//      four primitives on both sides, HLLC of the reconstructed states, HLLE
//      of the two cell averages, Ducros blend,
//   3. per cell: flux divergence, the SSP-RK3 combination with U0, c2p and
//      floors, stores the result into the interior and into every ghost cell
//      that mirrors it (so no separate boundary pass exists), and
//   4. in stage 3, max-reduces |u|+|v|+c of the new state into the grid's
//      step control for the next dt.
// This replaces compute_rhs + rk3_sX + apply_bc (+ reduce_max after stage 3)
// of fv_up7_ducros_2d.cu:370-612, three launches per stage and a host sync
// per step, by one launch per stage and none.
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

struct TileCtl {
    double dt;
    int run;    // compute the stage on this tile
    int copy;   // F32C stage 3 of a skipped step: carry the state across
};

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

template <int PREC, int ORDER, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, 1) stage_kernel(const StageArgs a)
{
    using R = typename PrecT<PREC>::R;
    using RR = typename PrecT<PREC>::RR;
    constexpr int G = (ORDER + 1) / 2;
    constexpr int SW = TX + 2 * G, SH = TY + 2 * G;
    constexpr int NXF = (TX + 1) * TY, NYF = TX * (TY + 1);
    constexpr int NW = NT / 32;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *S = reinterpret_cast<R *>(smem_raw);  // [4][SH][SW] primitives
    R *FX = S + 4 * SH * SW;                 // [4][TY][TX+1]
    R *FY = FX + 4 * TY * (TX + 1);          // [4][TY+1][TX]
    __shared__ TileCtl s_ctl;
    __shared__ double s_red[NW];

    const int tid = threadIdx.x;
    const bool batched = (a.grids != nullptr);
    const int ntiles = batched ? *a.ntiles : a.ntiles_static;

    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        GridDev gd;
        int tile;
        if (batched) {
            TileRef tr = a.tiles[t];
            gd = a.grids[tr.grid];
            tile = tr.tile;
        } else {
            gd = a.grid;
            tile = t;
        }
        const int n = gd.n;
        const int tx0 = (tile % gd.tiles_x) * TX, ty0 = (tile / gd.tiles_x) * TY;
        if (tid == 0) s_ctl = tile_control<PREC>(gd.ctrl, a.stage, tile == 0);
        __syncthreads();
        const TileCtl ctl = s_ctl;
        const Gas<R> gs{R(gd.gam), R(gd.gam) - R(1)};
        const int cur = a.parity, nxt = a.parity ^ 1;

        if (!ctl.run) {
            if constexpr (PREC == P32C) if (ctl.copy) {
                // skipped F32C step: the next step reads the other buffer
                const float *hi = (const float *)gd.st[cur], *lo = (const float *)gd.lo[cur];
                for (int k = tid; k < TX * TY; k += NT) {
                    int r = k / TX, c = k - r * TX, i = tx0 + c, j = ty0 + r;
                    if (i >= n || j >= n) continue;
                    float vh[4], vl[4];
                    long long e = gidx(gd, 0, j, i);
                    for (int q = 0; q < 4; ++q) { vh[q] = hi[e + q * gd.plane]; vl[q] = lo[e + q * gd.plane]; }
                    put_cell<float>(gd, (float *)gd.st[nxt], j, i, vh);
                    put_cell<float>(gd, (float *)gd.lo[nxt], j, i, vl);
                }
            }
            __syncthreads();
            continue;
        }
        const R dt = R(ctl.dt);
        const R inv_h = R(1.0 / gd.h);

        // ---- 1. halo tile -> shared memory (primitives) ----------------
        {
            const int np = n + 2 * G;
            const R *src;
            const float *inc = nullptr;
            if constexpr (PREC == P32C) {
                src = (const R *)gd.st[cur];
                if (a.stage == 2) inc = (const float *)gd.k1;
                else if (a.stage == 3) inc = (const float *)gd.k2;
            } else {
                src = (const R *)(a.stage == 2 ? gd.k1 : a.stage == 3 ? gd.k2 : gd.st[0]);
            }
            for (int k = tid; k < SH * SW; k += NT) {
                int r = k / SW, c = k - r * SW;
                int jp = ty0 + r, ip = tx0 + c;  // padded coordinates
                R w[4] = {R(0), R(0), R(0), R(0)};
                if (jp < np && ip < np) {
                    long long e = (long long)jp * gd.pitch + ip + gd.xoff;
                    if constexpr (PREC == P32C) {
                        float u[4];
                        for (int q = 0; q < 4; ++q) u[q] = __ldg(src + e + q * gd.plane);
                        if (inc)
                            for (int q = 0; q < 4; ++q) u[q] += __ldg(inc + e + q * gd.plane);
                        c2p<float>(u, w, gs);
                    } else {
                        for (int q = 0; q < 4; ++q) w[q] = __ldg(src + e + q * gd.plane);
                    }
                }
                for (int q = 0; q < 4; ++q) S[q * SH * SW + k] = w[q];
            }
        }
        __syncthreads();

        // ---- 2. face fluxes -------------------------------------------
        for (int f = tid; f < NXF + NYF; f += NT) {
            const bool xf = f < NXF;
            int r, c, st;
            if (xf) { r = f / (TX + 1); c = f - r * (TX + 1); st = 1; }
            else { int f2 = f - NXF; r = f2 / TX; c = f2 - r * TX; st = SW; }
            const int base = (r + G) * SW + (c + G);  // cell on the right/top of the face
            const int qn = xf ? 1 : 2, qt = xf ? 2 : 1;
            const int qs[4] = {0, qn, qt, 3};
            R L[4], Rv[4], WL[4], WR[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const R *v = S + qs[m] * SH * SW + base;
                R s[2 * G];
#pragma unroll
                for (int d = 0; d < 2 * G; ++d) s[d] = v[(d - G) * st];
                upface<R, RR, ORDER>(s, L[m], Rv[m]);
                WL[m] = s[G - 1];
                WR[m] = s[G];
            }
            L[0] = floor14(L[0]); Rv[0] = floor14(Rv[0]);
            L[3] = floor14(L[3]); Rv[3] = floor14(Rv[3]);
            R Fh[4], Fl[4];
            hllc<R>(L, Rv, Fh, gs);
            hlle<R>(WL, WR, Fl, gs);
            const R sd = ducros<R>(WL[3], WR[3]);
            const R one_m = R(1) - sd;
            R Fn[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) Fn[q] = one_m * Fh[q] + sd * Fl[q];
            if (xf) {
                R *o = FX + r * (TX + 1) + c;
                o[0] = Fn[0]; o[TY * (TX + 1)] = Fn[1]; o[2 * TY * (TX + 1)] = Fn[2]; o[3 * TY * (TX + 1)] = Fn[3];
            } else {
                R *o = FY + r * TX + c;
                o[0] = Fn[0]; o[(TY + 1) * TX] = Fn[2]; o[2 * (TY + 1) * TX] = Fn[1]; o[3 * (TY + 1) * TX] = Fn[3];
            }
        }
        __syncthreads();

        // ---- 3. divergence, RK combination, stores ----------------------
        double lmax = 0.0;
        for (int k = tid; k < TX * TY; k += NT) {
            int r = k / TX, c = k - r * TX, i = tx0 + c, j = ty0 + r;
            if (i >= n || j >= n) continue;
            R res[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const R *fx = FX + q * TY * (TX + 1) + r * (TX + 1) + c;
                const R *fy = FY + q * (TY + 1) * TX + r * TX + c;
                res[q] = -(fx[1] - fx[0]) * inv_h - (fy[TX] - fy[0]) * inv_h;
            }
            const int sc = (r + G) * SW + (c + G);
            if (a.stage == 0) {
                R *rhs = (R *)a.rhs;
                size_t n2 = (size_t)n * n, kk = (size_t)j * n + i;
                for (int q = 0; q < 4; ++q) rhs[q * n2 + kk] = res[q];
                R lam = dabs<R>(S[SH * SW + sc]) + dabs<R>(S[2 * SH * SW + sc]) + sound<R>(S[3 * SH * SW + sc], S[sc], gs);
                ((R *)a.lam)[kk] = lam;
                continue;
            }
            if constexpr (PREC == P32C) {
                const long long e = gidx(gd, 0, j, i);
                if (a.stage == 1) {
                    float d[4];
                    for (int q = 0; q < 4; ++q) d[q] = dt * res[q];
                    put_cell<float>(gd, (float *)gd.k1, j, i, d);
                } else if (a.stage == 2) {
                    const float *d1 = (const float *)gd.k1;
                    float d[4];
                    for (int q = 0; q < 4; ++q) d[q] = 0.25f * (d1[e + q * gd.plane] + dt * res[q]);
                    put_cell<float>(gd, (float *)gd.k2, j, i, d);
                } else {
                    const float *d2 = (const float *)gd.k2;
                    const float *hi = (const float *)gd.st[cur], *lo = (const float *)gd.lo[cur];
                    float vh[4], vl[4];
                    for (int q = 0; q < 4; ++q) {
                        float d = (2.0f / 3.0f) * (d2[e + q * gd.plane] + dt * res[q]);
                        vh[q] = hi[e + q * gd.plane];
                        vl[q] = lo[e + q * gd.plane];
                        df_add(vh[q], vl[q], d);
                    }
                    // floors rho, p >= 1e-14 on the new state
                    float w[4];
                    c2p<float>(vh, w, gs);
                    if (!(w[0] > 1e-14f)) { vh[0] = 1e-14f; vl[0] = 0.f; w[0] = 1e-14f; }
                    if (!(w[3] > 1e-14f)) {
                        float ke = 0.5f * (vh[1] * vh[1] + vh[2] * vh[2]) / vh[0];
                        vh[3] = 1e-14f / gs.gm1 + ke; vl[3] = 0.f; w[3] = 1e-14f;
                    }
                    put_cell<float>(gd, (float *)gd.st[nxt], j, i, vh);
                    put_cell<float>(gd, (float *)gd.lo[nxt], j, i, vl);
                    float lam = fabsf(vh[1] / vh[0]) + fabsf(vh[2] / vh[0]) + sound<float>(w[3], w[0], gs);
                    lmax = fmax(lmax, (double)lam);
                }
                continue;
            } else {
            // primitive-state modes (F64 / F32): the reference's update
            R wk[4], w0[4], c0[4], cv[4], w[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) wk[q] = S[q * SH * SW + sc];
            if (a.stage == 1) {
#pragma unroll
                for (int q = 0; q < 4; ++q) w0[q] = wk[q];
            } else {
                const R *u0 = (const R *)gd.st[0];
                const long long e = gidx(gd, 0, j, i);
#pragma unroll
                for (int q = 0; q < 4; ++q) w0[q] = u0[e + q * gd.plane];
            }
            p2c<R>(w0, c0, gs);
            if (a.stage == 1) {
#pragma unroll
                for (int q = 0; q < 4; ++q) cv[q] = c0[q] + dt * res[q];
            } else {
                R ck[4];
                p2c<R>(wk, ck, gs);
                if (a.stage == 2) {
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        cv[q] = FVB_LIT(R, 0.75) * c0[q] + FVB_LIT(R, 0.25) * (ck[q] + dt * res[q]);
                } else {
                    const R a3 = FVB_LIT(R, 1.) / FVB_LIT(R, 3.), b3 = FVB_LIT(R, 2.) / FVB_LIT(R, 3.);
#pragma unroll
                    for (int q = 0; q < 4; ++q) cv[q] = a3 * c0[q] + b3 * (ck[q] + dt * res[q]);
                }
            }
            c2p<R>(cv, w, gs);
            w[0] = floor14(w[0]);
            w[3] = floor14(w[3]);
            R *out = (R *)(a.stage == 1 ? gd.k1 : a.stage == 2 ? gd.k2 : gd.st[0]);
            put_cell<R>(gd, out, j, i, w);
            if (a.stage == 3) {
                R lam = dabs<R>(w[1]) + dabs<R>(w[2]) + sound<R>(w[3], w[0], gs);
                lmax = fmax(lmax, (double)lam);
            }
            }
        }

        // ---- 4. max wave speed of the new state (stage 3) ----------------
        if (a.stage == 3) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
            if ((tid & 31) == 0) s_red[tid >> 5] = lmax;
            __syncthreads();
            if (tid == 0) {
                double m = 0.0;
                for (int w = 0; w < NW; ++w) m = fmax(m, s_red[w]);
                atomicMax(&gd.ctrl->lam_acc, (unsigned long long)__double_as_longlong(m));
                if (tile == 0) leader_finish<PREC>(gd.ctrl);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// instantiation table
// ---------------------------------------------------------------------------
template <int PREC, int ORDER, int SHAPE>
struct K {
    static constexpr TileShape ts = kTileShapes[SHAPE];
    static constexpr int G = (ORDER + 1) / 2;
    using R = typename PrecT<PREC>::R;
    static size_t smem()
    {
        return sizeof(R) * (4 * (ts.ty + 2 * G) * (ts.tx + 2 * G) + 4 * ts.ty * (ts.tx + 1) + 4 * (ts.ty + 1) * ts.tx);
    }
    static void *fn() { return (void *)stage_kernel<PREC, ORDER, ts.tx, ts.ty, ts.nt>; }
};

struct KernelEntry {
    void *fn;
    size_t smem;
    int nt;
    int ready;
    int max_ctas;
};

template <int PREC, int ORDER, int SHAPE>
static KernelEntry entry()
{
    return KernelEntry{K<PREC, ORDER, SHAPE>::fn(), K<PREC, ORDER, SHAPE>::smem(),
                       kTileShapes[SHAPE].nt, 0, 0};
}

#define FVB_SHAPES(P, O) entry<P, O, 0>(), entry<P, O, 1>(), entry<P, O, 2>(), entry<P, O, 3>()

static KernelEntry *table_for(int prec, int order)
{
    static KernelEntry t64_7[] = {FVB_SHAPES(P64, 7)};
    static KernelEntry t64_5[] = {FVB_SHAPES(P64, 5)};
    static KernelEntry t64_3[] = {FVB_SHAPES(P64, 3)};
    static KernelEntry t32_7[] = {FVB_SHAPES(P32, 7)};
    static KernelEntry t32c_7[] = {FVB_SHAPES(P32C, 7)};
    if (prec == P64) return order == 7 ? t64_7 : order == 5 ? t64_5 : order == 3 ? t64_3 : nullptr;
    if (order != 7) return nullptr;
    return prec == P32 ? t32_7 : prec == P32C ? t32c_7 : nullptr;
}

static cudaError_t prepare(KernelEntry &e)
{
    if (e.ready) return cudaSuccess;
    cudaError_t err = cudaFuncSetAttribute(e.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)e.smem);
    if (err != cudaSuccess) return err;
    int nb = 0;
    err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, e.fn, e.nt, e.smem);
    if (err != cudaSuccess) return err;
    e.max_ctas = nb;
    e.ready = 1;
    return cudaSuccess;
}

size_t stage_smem_bytes(int prec, int order, int shape)
{
    KernelEntry *t = table_for(prec, order);
    return t ? t[shape].smem : 0;
}

int stage_max_ctas_per_sm(int prec, int order, int shape)
{
    KernelEntry *t = table_for(prec, order);
    if (!t || shape < 0 || shape >= kNumTileShapes) return 0;
    if (prepare(t[shape]) != cudaSuccess) return 0;
    return t[shape].max_ctas;
}

cudaError_t launch_stage(int prec, int order, int shape, const StageArgs &a, int grid_ctas, cudaStream_t s)
{
    KernelEntry *t = table_for(prec, order);
    if (!t || shape < 0 || shape >= kNumTileShapes) return cudaErrorInvalidValue;
    KernelEntry &e = t[shape];
    cudaError_t err = prepare(e);
    if (err != cudaSuccess) return err;
    if (grid_ctas <= 0) return cudaSuccess;
    void *args[] = {(void *)&a};
    return cudaLaunchKernel(e.fn, dim3(grid_ctas), dim3(e.nt), args, e.smem, s);
}

}  // namespace fvb
