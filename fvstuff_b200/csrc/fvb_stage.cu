// fvb_stage.cu -- the fused SSP-RK3 stage kernel of the FP64 plain method
// (and of the FP32 form as shipped), the step-control kernel of batched
// launches, the tile-variant tables and the TMA descriptors.  The FP32-
// compensated form has its own kernel (fvb_stage32c.cu).
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
#include <stdint.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include "fvb_internal.h"
#include "fvb_physics.cuh"
#include "fvb_device.cuh"
#include "fvb_tma.cuh"

namespace fvb {

// Flux through one face of the working tile W ([6][SH][SW]: rho, u, v, p,
// c, E) whose right/top cell is at `base`; XDIR: x-face (normal u), else
// y-face (normal v).  Writes the 4 Cartesian components to out[q * ostride].
template <int PREC, int ORDER, int SW, int PL, bool XDIR, int RS, class R>
__device__ __forceinline__ void face_one(const R *W, int base, R *out, int ostride, const GasF<R> &gf,
                                         const Gas<R> &gs)
{
    using RR = typename PrecT<PREC>::RR;
    constexpr int G = (ORDER + 1) / 2;
    constexpr int ST = XDIR ? 1 : SW;
    constexpr int QN = XDIR ? 1 : 2, QT = XDIR ? 2 : 1;
    constexpr int QS[4] = {0, QN, QT, 3};
    R L[4], Rv[4], WL[4], WR[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const R *v = W + QS[m] * PL + base;
        R s[2 * G];
#pragma unroll
        for (int d = 0; d < 2 * G; ++d) s[d] = v[(d - G) * ST];
        if constexpr (PREC != P32) upface_fast<R, ORDER>(s, L[m], Rv[m]);
        else upface<R, RR, ORDER>(s, L[m], Rv[m]);
        WL[m] = s[G - 1];
        WR[m] = s[G];
    }
    L[0] = floor14(L[0]); Rv[0] = floor14(Rv[0]);
    L[3] = floor14(L[3]); Rv[3] = floor14(Rv[3]);
    R Fn[4];
    if constexpr (PREC != P32) {
        const R *CE = W + 4 * PL + base;
        face_flux_fast<R, RS>(L, Rv, WL, WR, CE[-ST], CE[0], CE[PL - ST], CE[PL], gf, Fn);
    } else {
        R Fh[4], Fl[4];
        hllc<R, !XDIR>(L, Rv, Fh, gs);
        hlle<R, !XDIR>(WL, WR, Fl, gs);
        const R sd = ducros<R>(WL[3], WR[3]);
        const R one_m = R(1) - sd;
#pragma unroll
        for (int q = 0; q < 4; ++q) Fn[q] = one_m * Fh[q] + sd * Fl[q];
    }
    out[0] = Fn[0];
    out[ostride] = Fn[QN];
    out[2 * ostride] = Fn[QT];
    out[3 * ostride] = Fn[3];
}

// The FP64 and FP32 (reference-rounding) stage kernel, two CTAs per SM; the
// FP32-compensated form has its own kernel (fvb_stage32c.cu).
template <int PREC, int ORDER, int TX, int TY, int NT, bool BATCHED, int MINB, int RS>
__global__ void __launch_bounds__(NT, MINB) stage_kernel(const __grid_constant__ StageArgs a)
{
    static_assert(PREC == P64 || PREC == P32, "FP64 and FP32 primitive-state forms");
    using R = typename PrecT<PREC>::R;
    using RR = typename PrecT<PREC>::RR;
    constexpr int G = (ORDER + 1) / 2;
    constexpr int SW = TX + 2 * G, SH = TY + 2 * G, PL = SW * SH;
    constexpr int NXF = (TX + 1) * TY, NYF = TX * (TY + 1);
    constexpr int NW = NT / 32;
    // the throughput paths keep each cell's sound speed and energy too
    constexpr bool FAST = (PREC != P32);
    // IN: the tile as loaded (TMA lands here); W: primitives (+ c, E) the
    // faces are computed from, so IN can take the next tile meanwhile
    extern __shared__ __align__(128) unsigned char smem_raw[];
    R *IN = reinterpret_cast<R *>(smem_raw);
    R *W = IN + 4 * PL;
    R *FX = W + 6 * PL;               // [4][TY][TX+1]
    R *FY = FX + 4 * TY * (TX + 1);   // [4][TY+1][TX]
    __shared__ double s_red[NW];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ int s_err;
    __shared__ __align__(16) TileHdr s_hdr[2];
    __shared__ TileRef s_ref_next;  // batched: table entry of the CTA's next tile

    const int tid = threadIdx.x;
    constexpr bool batched = BATCHED;
    const int ntiles = batched ? *a.ntiles : a.ntiles_static;
    const int cur = a.parity;
    if (tid == 0) {
        mbar_init(&s_bar, 1);
        s_err = 0;
    }
    __syncthreads();

    // every thread waits on the mbarrier itself (the completed phase makes the
    // TMA bytes visible to it); the barrier after the wait also agrees on s_err
    uint32_t phase = 0;
    auto wait_box = [&](bool tma) {
        if (tma) {
            if (mbar_wait(&s_bar, phase)) phase ^= 1;
            else s_err = 1;
        }
        __syncthreads();
    };
    // single grid: start the halo-box load of tile t (every thread: the
    // plain path loads cooperatively)
    auto start_single = [&](int t) -> bool {
        if (tid == 0 && a.grid.tmap) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue_tile_load<PREC, G, SW, SH, NT>(a.grid, a.stage, cur, t, IN, &s_bar, tid);
        return a.grid.tmap != nullptr;
    };
    // failure injection (fvb_debug_drop_load): CTA 0 of a single-grid launch
    // issues no first box load, so its bounded wait runs out and the grid's
    // status becomes FVB_ERR_TIMEOUT; the flag is read by every thread of
    // that CTA before thread 0 clears it behind the first barrier
    const bool drop = !batched && blockIdx.x == 0 && a.stage > 0 && a.grid.ctrl && a.grid.tmap &&
                      *(volatile int *)&a.grid.ctrl->drop_load;
    const int stride = gridDim.x;
    int t = blockIdx.x, slot = 0;
    if (t < ntiles && batched) {
        if (tid < 32) {
            const TileRef r0 = a.tiles[t];
            start_batched_tile<PREC, G, SW, SH, NT>(a, &s_hdr[0], r0, hdr_word(a, r0, tid), cur, IN, &s_bar, tid);
            if (tid == 0 && t + stride < ntiles) s_ref_next = a.tiles[t + stride];
        }
        wait_box(true);
    } else if (drop) {
        wait_box(true);  // nothing was issued: the wait runs out
        if (tid == 0) a.grid.ctrl->drop_load = 0;
    } else {
        wait_box(t < ntiles ? start_single(t) : false);
    }
    // which of this thread's conversion cells (k = tid + it NT) the HLLE
    // reads the sound speed and energy of: the interior rows x columns
    // [G-1, G+TX], and rows G-1, G+TY x the interior columns (the same cells
    // in every tile, so the mask is formed once)
    constexpr int NCV = (PL + NT - 1) / NT;
    static_assert(NCV <= 32, "one mask bit per conversion cell");
    unsigned cemask = 0;
#pragma unroll
    for (int it = 0; it < NCV; ++it) {
        const int k = tid + it * NT, r = k / SW, c = k - r * SW;
        const bool ce = ((unsigned)(r - G) < (unsigned)TY && (unsigned)(c - (G - 1)) < (unsigned)(TX + 2)) ||
                        ((r == G - 1 || r == G + TY) && (unsigned)(c - G) < (unsigned)TX);
        cemask |= (ce && k < PL ? 1u : 0u) << it;
    }
    // single grid: the stage-3 wave-speed max is reduced once per CTA, and the
    // step control, the same for every tile, is read once (the leader is CTA
    // 0, whose first tile is tile 0)
    double lacc = 0.0;
    TileCtl ctl1{};
    if (!batched && t < ntiles) ctl1 = tile_control<PREC>(a.grid.ctrl, a.stage, tid == 0 && t == 0);
    for (; t < ntiles; t += stride, slot ^= 1) {
        // warp 0 of a batched launch: the next tile's descriptor word and the
        // entry of the tile after it, in flight during the conversion
        const bool has_next = t + stride < ntiles;
        unsigned long long wnext = 0ull;
        TileRef ref_next{}, ref_after{};
        if (batched && tid < 32) {
            if (has_next) {
                ref_next = s_ref_next;
                wnext = hdr_word(a, ref_next, tid);
            }
            if (t + 2 * stride < ntiles) ref_after = a.tiles[t + 2 * stride];
        }
        const GridDev &gd = tile_grid<BATCHED>(s_hdr[slot], a);
        const int tile = batched ? s_hdr[slot].tile : t;
        const TileCtl ctl = batched ? s_hdr[slot].ctl : ctl1;
        const int n = gd.n;
        const int tx0 = (tile % gd.tiles_x) * TX, ty0 = (tile / gd.tiles_x) * TY;
        const Gas<R> gs{R(gd.gam), R(gd.gam) - R(1)};
        const GasF<R> gf{R(gd.gam), R(1.0 / (gd.gam - 1.0)), R(gd.gam) - R(1)};
        if (s_err) {
            // a halo load never arrived: record it, skip the tile
            if (tid == 0 && gd.ctrl) gd.ctrl->status = FVB_ERR_TIMEOUT;
            break;
        }
        if (ctl.run && a.stage >= 0) {
#pragma unroll
            for (int it = 0; it < NCV; ++it) {
                const int k = tid + it * NT;
                if (k >= PL) break;
                R w0 = IN[k], w1 = IN[PL + k], w2 = IN[2 * PL + k], w3 = IN[3 * PL + k];
                if constexpr (FAST) {
                    if ((cemask >> it) & 1u) {
                        R cc, ee;
                        cell_ce<R>(w0, w1, w2, w3, gf, cc, ee);
                        W[4 * PL + k] = cc;
                        W[5 * PL + k] = ee;
                    }
                }
                W[k] = w0; W[PL + k] = w1; W[2 * PL + k] = w2; W[3 * PL + k] = w3;
            }
        }
        __syncthreads();
        // ---- 2. load the next tile into IN (asynchronous through TMA) -------
        // (the fence orders this CTA's reads of IN before the async-proxy
        // writes; in a batched launch warp 0 also fetches that tile's header)
        bool next_tma = false;
        if (has_next) {
            if (batched) {
                if (tid < 32) {
                    start_batched_tile<PREC, G, SW, SH, NT>(a, &s_hdr[slot ^ 1], ref_next, wnext, cur, IN, &s_bar,
                                                            tid);
                    if (tid == 0) s_ref_next = ref_after;
                }
                next_tma = true;
            } else {
                next_tma = start_single(t + stride);
            }
        }

        if (!ctl.run) {
            wait_box(next_tma);
            continue;
        }
        const R dt = R(ctl.dt);
        const R inv_h = R(1.0 / gd.h);
        const R hR = R(gd.h);  // the FP32 form divides by h, as the shipped solver does
        // U0 of this thread's cells (stages 2 and 3), loaded now so the loads
        // are in flight while the faces are computed
        constexpr int CPT = (TX * TY + NT - 1) / NT;  // cells per thread
        static_assert(CPT <= 2, "at most two cells a thread");
        R u0v[CPT][4];
        if (a.stage >= 2) {
            const R *u0 = (const R *)gd.st[0];
#pragma unroll
            for (int it = 0; it < CPT; ++it) {
                const int k = tid + it * NT, r = k / TX, c = k - r * TX, i = tx0 + c, j = ty0 + r;
                if (k < TX * TY && i < n && j < n) {
                    const long long e = gidx(gd, 0, j, i);
#pragma unroll
                    for (int q = 0; q < 4; ++q) u0v[it][q] = u0[e + q * gd.plane];
                }
            }
        }

        // ---- 3. face fluxes: x-faces, then y-faces (compile-time strides) ---
        for (int f = tid; f < NXF; f += NT) {
            const int r = f / (TX + 1), c = f - r * (TX + 1);
            face_one<PREC, ORDER, SW, PL, true, RS>(W, (r + G) * SW + (c + G), FX + r * (TX + 1) + c, TY * (TX + 1),
                                               gf, gs);
        }
        for (int f = tid; f < NYF; f += NT) {
            const int r = f / TX, c = f - r * TX;
            face_one<PREC, ORDER, SW, PL, false, RS>(W, (r + G) * SW + (c + G), FY + r * TX + c, (TY + 1) * TX, gf,
                                                gs);
        }
        __syncthreads();

        // ---- 4. divergence, RK combination, stores ------------------------
        double lmax = 0.0;
#pragma unroll
        for (int it = 0; it < CPT; ++it) {
            const int k = tid + it * NT;
            if (k >= TX * TY) break;
            int r = k / TX, c = k - r * TX, i = tx0 + c, j = ty0 + r;
            if (i >= n || j >= n) continue;
            R res[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const R *fx = FX + q * TY * (TX + 1) + r * (TX + 1) + c;
                const R *fy = FY + q * (TY + 1) * TX + r * TX + c;
                if constexpr (FAST) res[q] = -(fx[1] - fx[0]) * inv_h - (fy[TX] - fy[0]) * inv_h;
                else res[q] = -(fx[1] - fx[0]) / hR - (fy[TX] - fy[0]) / hR;  // fv_up7_ducros_2d.cu:500-503
            }
            const int sc = (r + G) * SW + (c + G);
            if (a.stage == 0) {
                R *rhs = (R *)a.rhs;
                size_t n2 = (size_t)n * n, kk = (size_t)j * n + i;
                for (int q = 0; q < 4; ++q) rhs[q * n2 + kk] = res[q];
                ((R *)a.lam)[kk] = dabs<R>(W[PL + sc]) + dabs<R>(W[2 * PL + sc]) + sound<R>(W[3 * PL + sc], W[sc], gs);
                continue;
            }
            {
                // primitive-state modes (F64 / F32): the reference's update
                R wk[4], w0[4], c0[4], cv[4], w[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) wk[q] = W[q * PL + sc];
                if (a.stage == 1) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) w0[q] = wk[q];
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) w0[q] = u0v[it][q];
                }
                if constexpr (FAST) {
                    c0[0] = w0[0]; c0[1] = w0[0] * w0[1]; c0[2] = w0[0] * w0[2];
                    c0[3] = w0[3] * gf.igm1 + R(0.5) * w0[0] * (w0[1] * w0[1] + w0[2] * w0[2]);
                } else {
                    p2c<R>(w0, c0, gs);
                }
                if (a.stage == 1) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) cv[q] = c0[q] + dt * res[q];
                } else {
                    R ck[4];
                    if constexpr (FAST) {
                        ck[0] = wk[0]; ck[1] = wk[0] * wk[1]; ck[2] = wk[0] * wk[2];
                        ck[3] = wk[3] * gf.igm1 + R(0.5) * wk[0] * (wk[1] * wk[1] + wk[2] * wk[2]);
                    } else {
                        p2c<R>(wk, ck, gs);
                    }
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
                if constexpr (FAST) {
                    const R ir = frcp(cv[0]);
                    w[0] = cv[0];
                    w[1] = cv[1] * ir;
                    w[2] = cv[2] * ir;
                    w[3] = gf.gm1 * (cv[3] - R(0.5) * (cv[1] * cv[1] + cv[2] * cv[2]) * ir);
                } else {
                    c2p<R>(cv, w, gs);
                }
                w[0] = floor14(w[0]);
                w[3] = floor14(w[3]);
                R *out = (R *)(a.stage == 1 ? gd.k1 : a.stage == 2 ? gd.k2 : gd.st[0]);
                put_cell<R>(gd, out, j, i, w);
                if (a.stage == 3) {
                    R lam;
                    if constexpr (FAST) {
                        R c;
                        if constexpr (sizeof(R) == 8) {
                            c = snd_rsq(gf.gam * w[3], w[0]);
                        } else {
                            R cs2 = gf.gam * w[3] * frcp(w[0]);
                            c = fsqrt(cs2 > FVB_LIT(R, 1e-14) ? cs2 : FVB_LIT(R, 1e-14));
                        }
                        lam = dabs<R>(w[1]) + dabs<R>(w[2]) + c;
                    } else {
                        lam = dabs<R>(w[1]) + dabs<R>(w[2]) + sound<R>(w[3], w[0], gs);
                    }
                    // (a NaN lam is skipped, as fmax skips it; one compare-select)
                    lmax = smax<double>((double)lam, lmax);
                }
            }
        }

        // ---- 5. max wave speed of the new state (stage 3) ------------------
        if (a.stage == 3) {
            // (a batched launch advances each grid's time where its tile 0's header is published)
            if (!batched && tid == 0 && tile == 0) leader_finish<PREC>(gd.ctrl);
            if (batched) {
                // tiles of one CTA belong to different grids: one atomic per
                // warp and tile
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
                if ((tid & 31) == 0 && lmax > 0.0)
                    atomicMax(&gd.ctrl->lam_acc, (unsigned long long)__double_as_longlong(lmax));
            } else {
                lacc = fmax(lacc, lmax);
            }
        }
        // ---- 6. next tile's halo box: wait, then release W / FX / FY -------
        wait_box(next_tma);
    }
    if (!batched && a.stage == 3) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) lacc = fmax(lacc, __shfl_xor_sync(0xffffffffu, lacc, o));
        if ((tid & 31) == 0) s_red[tid >> 5] = lacc;
        __syncthreads();
        if (tid == 0 && a.grid.ctrl) {
            double m = 0.0;
            for (int w = 0; w < NW; ++w) m = fmax(m, s_red[w]);
            if (m > 0.0) atomicMax(&a.grid.ctrl->lam_acc, (unsigned long long)__double_as_longlong(m));
        }
    }
    // a load still in flight after an error: wait for it (bounded) so no
    // copy into this CTA's shared memory outlives it
    if (s_err && gd_has_tma(a)) mbar_wait(&s_bar, phase);
}

// ---------------------------------------------------------------------------
// instantiation table
// ---------------------------------------------------------------------------
template <int PREC, int ORDER, int SHAPE, int RS = 0>
struct K {
    static constexpr TileShape ts = kTileShapes[SHAPE];
    static constexpr int G = (ORDER + 1) / 2;
    using R = typename PrecT<PREC>::R;
    static constexpr size_t kSmem = sizeof(R) * (10 * (ts.ty + 2 * G) * (ts.tx + 2 * G) + 4 * ts.ty * (ts.tx + 1) +
                                                 4 * (ts.ty + 1) * ts.tx);
    // CTAs per SM the registers are budgeted for: three where three tiles'
    // shared memory fits in the SM's 228 KB (1 KB reserved per CTA), else two
    static constexpr int kMinBlocks = 3 * (kSmem + 1024) <= 228 * 1024 ? 3 : 2;
    static size_t smem() { return kSmem; }
    static void *fn() { return (void *)stage_kernel<PREC, ORDER, ts.tx, ts.ty, ts.nt, false, kMinBlocks, RS>; }
    static void *fn_batched() { return (void *)stage_kernel<PREC, ORDER, ts.tx, ts.ty, ts.nt, true, kMinBlocks, RS>; }
};

struct KernelEntry {
    void *fn;          // single grid
    void *fn_batched;  // tile table
    size_t smem;
    int nt;
};

template <int PREC, int ORDER, int SHAPE, int RS = 0>
static KernelEntry entry()
{
    using KK = K<PREC, ORDER, SHAPE, RS>;
    return KernelEntry{KK::fn(), KK::fn_batched(), KK::smem(), kTileShapes[SHAPE].nt};
}

static KernelEntry entry32c(int shape)
{
    return KernelEntry{stage32c_fn(shape, false), stage32c_fn(shape, true), stage32c_smem(shape),
                       kTileShapes[shape].nt};
}

#define FVB_SHAPES(P, O) \
    entry<P, O, 0>(), entry<P, O, 1>(), entry<P, O, 2>(), entry<P, O, 3>(), entry<P, O, 4>(), entry<P, O, 5>(), \
        entry<P, O, 6>()
#define FVB_SHAPES_RS(RS) \
    entry<P64, 7, 0, RS>(), entry<P64, 7, 1, RS>(), entry<P64, 7, 2, RS>(), entry<P64, 7, 3, RS>(), \
        entry<P64, 7, 4, RS>(), entry<P64, 7, 5, RS>(), entry<P64, 7, 6, RS>()

static KernelEntry *table_for(int prec, int order, int rs = 0)
{

    static KernelEntry t64_7_hll[] = {FVB_SHAPES_RS(1)};
    static KernelEntry t64_7_roe[] = {FVB_SHAPES_RS(2)};
    if (rs != 0) return (prec == P64 && order == 7) ? (rs == 1 ? t64_7_hll : rs == 2 ? t64_7_roe : nullptr) : nullptr;
    static KernelEntry t64_7[] = {FVB_SHAPES(P64, 7)};
    static KernelEntry t64_5[] = {FVB_SHAPES(P64, 5)};
    static KernelEntry t64_3[] = {FVB_SHAPES(P64, 3)};
    static KernelEntry t64_9[] = {FVB_SHAPES(P64, 9)};
    static KernelEntry t32_7[] = {FVB_SHAPES(P32, 7)};
    static KernelEntry t32c_7[] = {entry32c(0), entry32c(1), entry32c(2), entry32c(3), entry32c(4), entry32c(5),
                                   entry32c(6)};
    if (prec == P64)
        return order == 7 ? t64_7 : order == 5 ? t64_5 : order == 3 ? t64_3 : order == 9 ? t64_9 : nullptr;
    if (order != 7) return nullptr;
    return prec == P32 ? t32_7 : prec == P32C ? t32c_7 : nullptr;
}

cudaError_t launch_facts(const void *fn, int threads, size_t smem, LaunchFacts &out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::mutex mu;
    static std::map<std::tuple<const void *, int, int, size_t>, LaunchFacts> known;
    const auto key = std::make_tuple(fn, dev, threads, smem);
    std::lock_guard<std::mutex> lk(mu);
    const auto it = known.find(key);
    if (it != known.end()) {
        out = it->second;
        return cudaSuccess;
    }
    LaunchFacts f{};
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&f.ctas_per_sm, fn, threads, smem);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&f.sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    if (f.ctas_per_sm <= 0) return cudaErrorInvalidConfiguration;
    known.emplace(key, f);
    out = f;
    return cudaSuccess;
}

// resident CTAs per SM of a table entry: the fewer of its two kernels
static cudaError_t prepare(const KernelEntry &e, int &max_ctas)
{
    LaunchFacts a{}, b{};
    cudaError_t err = launch_facts(e.fn, e.nt, e.smem, a);
    if (err == cudaSuccess) err = launch_facts(e.fn_batched, e.nt, e.smem, b);
    if (err != cudaSuccess) return err;
    max_ctas = std::min(a.ctas_per_sm, b.ctas_per_sm);
    return cudaSuccess;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    // looked up once (a function-local static's initialisation is thread-safe)
    static const EncodeTiledFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return (EncodeTiledFn)p;
        return (EncodeTiledFn) nullptr;
    }();
    return fn;
}

// Descriptors of the (TX+2g) x (TY+2g) x 4 halo box of each padded buffer.
// The tensor is (x = memory column, y = padded row, z = variable plane);
// x starts at column 0 of the pitched row, so a tile's box starts at
// x = xoff + tx0.  Every such x, the pitch and the plane stride must be
// 16-byte multiples; out-of-range parts of ragged tiles are zero-filled.
bool encode_tile_maps(const GridDev &gd, int prec, int order, int shape, CUtensorMap out[TM_COUNT])
{
    EncodeTiledFn enc = encode_fn();
    if (!enc || shape < 0 || shape >= kNumTileShapes) return false;
    const TileShape &ts = kTileShapes[shape];
    const int g = (order + 1) / 2, np = gd.n + 2 * g;
    const size_t es = prec == P64 ? 8 : 4;
    const int sw = ts.tx + 2 * g, sh = ts.ty + 2 * g;
    if (((size_t)gd.pitch * es) % 16 || ((size_t)gd.plane * es) % 16 || ((size_t)gd.xoff * es) % 16 ||
        ((size_t)ts.tx * es) % 16 || ((size_t)sw * es) % 16 || sw > 256 || sh > 256)
        return false;
    cuuint64_t dims[3] = {(cuuint64_t)(gd.xoff + np), (cuuint64_t)np, 4};
    cuuint64_t strides[2] = {(cuuint64_t)gd.pitch * es, (cuuint64_t)gd.plane * es};
    cuuint32_t box[3] = {(cuuint32_t)sw, (cuuint32_t)sh, 4};
    cuuint32_t estr[3] = {1, 1, 1};
    void *bufs[TM_COUNT] = {gd.st[0], gd.st[1] ? gd.st[1] : gd.st[0], gd.k1, gd.k2};
    for (int m = 0; m < TM_COUNT; ++m) {
        if (((uintptr_t)bufs[m]) % 16) return false;
        CUresult r = enc(&out[m], es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
                         bufs[m], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                         CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return false;
    }
    return true;
}

// Copy a grid's tensor maps into device memory from a kernel parameter, so
// the host copy need not outlive the call (no stream synchronisation).
struct TileMaps {
    CUtensorMap m[TM_COUNT];
};

__global__ void put_maps_kernel(const __grid_constant__ TileMaps maps, CUtensorMap *dst)
{
    constexpr int NV = (int)(sizeof(TileMaps) / 16);
    const int k = threadIdx.x;
    if (k < NV) reinterpret_cast<uint4 *>(dst)[k] = reinterpret_cast<const uint4 *>(&maps)[k];
}

cudaError_t put_tile_maps(const CUtensorMap maps[TM_COUNT], CUtensorMap *dst, cudaStream_t s)
{
    static_assert(sizeof(TileMaps) % 16 == 0 && sizeof(TileMaps) / 16 <= 64, "one small block copies the maps");
    TileMaps tm;
    for (int m = 0; m < TM_COUNT; ++m) tm.m[m] = maps[m];
    put_maps_kernel<<<1, 64, 0, s>>>(tm, dst);
    return cudaGetLastError();
}

size_t stage_smem_bytes(int prec, int order, int shape, int rs)
{
    KernelEntry *t = table_for(prec, order, rs);
    return t ? t[shape].smem : 0;
}

int stage_max_ctas_per_sm(int prec, int order, int shape, int rs)
{
    KernelEntry *t = table_for(prec, order, rs);
    if (!t || shape < 0 || shape >= kNumTileShapes) return 0;
    int max_ctas = 0;
    if (prepare(t[shape], max_ctas) != cudaSuccess) return 0;
    return max_ctas;
}

cudaError_t launch_stage(int prec, int order, int shape, const StageArgs &a, int grid_ctas, cudaStream_t s, int rs)
{
    KernelEntry *t = table_for(prec, order, rs);
    if (!t || shape < 0 || shape >= kNumTileShapes) return cudaErrorInvalidValue;
    const KernelEntry &e = t[shape];
    int max_ctas = 0;
    cudaError_t err = prepare(e, max_ctas);
    if (err != cudaSuccess) return err;
    if (grid_ctas <= 0) return cudaSuccess;
    void *args[] = {(void *)&a};
    return cudaLaunchKernel(a.grids ? e.fn_batched : e.fn, dim3(grid_ctas), dim3(e.nt), args, e.smem, s);
}

}  // namespace fvb
