// fvb_stage64.cu -- the fused SSP-RK3 stage kernel of the FP64 plain method,
// laid out for three resident CTAs per SM.
//
// The FP64 stage is bound by the FP64 pipe and its latency, not by HBM: a
// cell-stage is ~550 FP64 instructions against 85 bytes of HBM traffic, so
// what sets the speed is how many warps an SM holds to cover the FP64 and
// shared-memory latencies.  This kernel keeps per CTA only what the tile
// needs at one time, so three 256-thread CTAs (24 warps) fit in an SM's
// 228 KB and 64K registers:
//   W    the (TX+2g) x (TY+2g) halo box of the stage input, 4 planes of
//        primitives -- the TMA lands here and the faces read it directly
//        (no separate landing buffer, no copy pass);
//   CE   sound speed and total energy of the (TX+2) x (TY+2) cells whose
//        states the HLLE of a tile face reads;
//   FX   x-face fluxes [4][TY][TX+1],  FY  y-face fluxes [4][TY+1][TX].
// A face is evaluated in three steps that each hold few registers -- the
// HLLE of the two cell states with the pressure-jump sensor, then the
// UP-ORDER reconstructions one variable at a time, then the solver on the
// reconstructed states and the blend -- with the same arithmetic as the
// two-CTA kernel (fvb_stage.cu).
//
// Per tile: wait for the box; per-cell c and E into CE; every face once;
// each thread takes its cells' stage input into registers; barrier; thread 0
// starts the next tile's box load, which then overlaps the divergence, the
// RK combination and the stores (interior + ghost images); stage 3
// max-reduces |u|+|v|+c of the new state for the next dt.  U0 (stages 2, 3)
// is prefetched into L2 when the tile starts.
//
// This replaces compute_rhs + rk3_sX + apply_bc (+ reduce_max after stage 3)
// of fv_up7_ducros_2d.cu:370-612.
#include <stdint.h>

#include "fvb_internal.h"
#include "fvb_physics.cuh"
#include "fvb_device.cuh"
#include "fvb_tma.cuh"

namespace fvb {

// Flux through one face of the box W ([4][SH][SW] primitives) whose
// right/top cell is at box index `base` and CE index `cb`; XDIR: x-face
// (normal u), else y-face (normal v).  Writes the 4 Cartesian components to
// out[q * ostride].
template <int ORDER, int SW, int PL, int CW, int CPL, bool XDIR, int RS>
__device__ __forceinline__ void face64(const double *W, const double *CE, int base, int cb, double *out, int ostride,
                                       const GasF<double> &gf)
{
    constexpr int G = (ORDER + 1) / 2;
    constexpr int ST = XDIR ? 1 : SW;   // box stride along the normal
    constexpr int CS = XDIR ? 1 : CW;   // CE stride along the normal
    constexpr int QN = XDIR ? 1 : 2, QT = XDIR ? 2 : 1;
    constexpr int QS[4] = {0, QN, QT, 3};
    // 1. HLLE of the two cell states and the sensor
    double Fl[4], sd;
    {
        double WL[4], WR[4];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            WL[m] = W[QS[m] * PL + base - ST];
            WR[m] = W[QS[m] * PL + base];
        }
        hlle_sensor_fast<double>(WL, WR, CE[cb - CS], CE[cb], CE[CPL + cb - CS], CE[CPL + cb], Fl, sd);
    }
    // 2. UP-ORDER reconstruction, one variable at a time, floors on rho, p
    double L[4], Rv[4];
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        const double *v = W + QS[m] * PL + base;
        double s[2 * G];
#pragma unroll
        for (int d = 0; d < 2 * G; ++d) s[d] = v[(d - G) * ST];
        upface_fast<double, ORDER>(s, L[m], Rv[m]);
    }
    L[0] = floor14(L[0]); Rv[0] = floor14(Rv[0]);
    L[3] = floor14(L[3]); Rv[3] = floor14(Rv[3]);
    // 3. solver on the reconstructed states, blend
    double Fh[4], Fn[4];
    recon_flux_fast<double, RS>(L, Rv, gf, Fh);
    ducros_blend<double>(Fh, Fl, sd, Fn);
    out[0] = Fn[0];
    out[ostride] = Fn[QN];
    out[2 * ostride] = Fn[QT];
    out[3 * ostride] = Fn[3];
}

template <int ORDER, int TX, int TY>
struct Lean64 {
    static constexpr int G = (ORDER + 1) / 2;
    static constexpr int SW = TX + 2 * G, SH = TY + 2 * G, PL = SW * SH;
    static constexpr int CW = TX + 2, CH = TY + 2, CPL = CW * CH;
    static constexpr size_t kSmem =
        sizeof(double) * ((size_t)4 * PL + 2 * CPL + 4 * TY * (TX + 1) + 4 * (TY + 1) * TX);
};

template <int ORDER, int TX, int TY, int NT, bool BATCHED, int MINB, int RS>
__global__ void __launch_bounds__(NT, MINB) stage64_kernel(const __grid_constant__ StageArgs a)
{
    using LY = Lean64<ORDER, TX, TY>;
    constexpr int G = LY::G, SW = LY::SW, SH = LY::SH, PL = LY::PL;
    constexpr int CW = LY::CW, CH = LY::CH, CPL = LY::CPL;
    constexpr int NXF = (TX + 1) * TY, NYF = TX * (TY + 1);
    constexpr int NW = NT / 32;
    constexpr int CPT = (TX * TY + NT - 1) / NT;  // cells per thread
    static_assert(CPT <= 2, "at most two cells a thread");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    double *W = reinterpret_cast<double *>(smem_raw);
    double *CE = W + 4 * PL;               // [2][CH][CW]: c, E
    double *FX = CE + 2 * CPL;             // [4][TY][TX+1]
    double *FY = FX + 4 * TY * (TX + 1);   // [4][TY+1][TX]
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

    uint32_t phase = 0;
    auto wait_box = [&](bool tma) {
        if (tma) {
            if (mbar_wait(&s_bar, phase)) phase ^= 1;
            else s_err = 1;
        }
        __syncthreads();
    };
    auto start_single = [&](int t) -> bool {
        if (tid == 0 && a.grid.tmap) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue_tile_load<P64, G, SW, SH, NT>(a.grid, a.stage, cur, t, W, &s_bar, tid);
        return a.grid.tmap != nullptr;
    };
    // failure injection (fvb_debug_drop_load), as in the two-CTA kernel
    const bool drop = !batched && blockIdx.x == 0 && a.stage > 0 && a.grid.ctrl && a.grid.tmap &&
                      *(volatile int *)&a.grid.ctrl->drop_load;
    const int stride = gridDim.x;
    int t = blockIdx.x, slot = 0;
    if (t < ntiles && batched) {
        if (tid < 32) {
            const TileRef r0 = a.tiles[t];
            start_batched_tile<P64, G, SW, SH, NT>(a, &s_hdr[0], r0, hdr_word(a, r0, tid), cur, W, &s_bar, tid);
            if (tid == 0 && t + stride < ntiles) s_ref_next = a.tiles[t + stride];
        }
        wait_box(true);
    } else if (drop) {
        wait_box(true);  // nothing was issued: the wait runs out
        if (tid == 0) a.grid.ctrl->drop_load = 0;
    } else {
        wait_box(t < ntiles ? start_single(t) : false);
    }
    double lacc = 0.0;
    TileCtl ctl1{};
    if (!batched && t < ntiles) ctl1 = tile_control<P64>(a.grid.ctrl, a.stage, tid == 0 && t == 0);
    for (; t < ntiles; t += stride, slot ^= 1) {
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
        const GasF<double> gf{gd.gam, 1.0 / (gd.gam - 1.0), gd.gam - 1.0};
        if (s_err) {
            if (tid == 0 && gd.ctrl) gd.ctrl->status = FVB_ERR_TIMEOUT;
            break;
        }
        const bool run = ctl.run && a.stage >= 0;
        if (run) {
            // U0 of this tile's cells into L2 (stages 2, 3): one prefetch
            // per 16-double line of each interior row and variable; a line
            // starting inside the interior ends inside the pitched row
            if (a.stage >= 2) {
                constexpr int LPR = (TX + 15) / 16;
                for (int k = tid; k < 4 * TY * LPR; k += NT) {
                    const int q = k / (TY * LPR), rem = k - q * (TY * LPR), r = rem / LPR, h = rem - r * LPR;
                    const int j = ty0 + r, i = tx0 + 16 * h;
                    if (j < n && i < n) {
                        const double *p = (const double *)gd.st[0] + gidx(gd, q, j, i);
                        asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
                    }
                }
            }
            // sound speed and energy of the cells the HLLE reads: rows
            // [G-1, G+TY] x columns [G-1, G+TX] of the box, without corners
            for (int k = tid; k < CPL; k += NT) {
                const int rr = k / CW, cc = k - rr * CW;
                if ((rr == 0 || rr == CH - 1) && (cc == 0 || cc == CW - 1)) continue;
                const int b = (rr + G - 1) * SW + (cc + G - 1);
                double c, e;
                cell_ce<double>(W[b], W[PL + b], W[2 * PL + b], W[3 * PL + b], gf, c, e);
                CE[k] = c;
                CE[CPL + k] = e;
            }
        }
        __syncthreads();
        // ---- faces: x, then y (compile-time strides) -----------------------
        if (run) {
            for (int f = tid; f < NXF; f += NT) {
                const int r = f / (TX + 1), c = f - r * (TX + 1);
                face64<ORDER, SW, PL, CW, CPL, true, RS>(W, CE, (r + G) * SW + (c + G), (r + 1) * CW + (c + 1),
                                                         FX + r * (TX + 1) + c, TY * (TX + 1), gf);
            }
            for (int f = tid; f < NYF; f += NT) {
                const int r = f / TX, c = f - r * TX;
                face64<ORDER, SW, PL, CW, CPL, false, RS>(W, CE, (r + G) * SW + (c + G), (r + 1) * CW + (c + 1),
                                                          FY + r * TX + c, (TY + 1) * TX, gf);
            }
        }
        // this thread's cells: stage input from the box, U0 from global
        double wk[CPT][4], u0v[CPT][4];
        if (run) {
#pragma unroll
            for (int it = 0; it < CPT; ++it) {
                const int k = tid + it * NT, r = k / TX, c = k - r * TX, i = tx0 + c, j = ty0 + r;
                if (k < TX * TY && i < n && j < n) {
                    const int sc = (r + G) * SW + (c + G);
#pragma unroll
                    for (int q = 0; q < 4; ++q) wk[it][q] = W[q * PL + sc];
                    if (a.stage >= 2) {
                        const double *u0 = (const double *)gd.st[0];
                        const long long e = gidx(gd, 0, j, i);
#pragma unroll
                        for (int q = 0; q < 4; ++q) u0v[it][q] = u0[e + q * gd.plane];
                    }
                }
            }
        }
        __syncthreads();
        // ---- the next tile's box into W, overlapping what follows ----------
        bool next_tma = false;
        if (has_next) {
            if (batched) {
                if (tid < 32) {
                    start_batched_tile<P64, G, SW, SH, NT>(a, &s_hdr[slot ^ 1], ref_next, wnext, cur, W, &s_bar,
                                                           tid);
                    if (tid == 0) s_ref_next = ref_after;
                }
                next_tma = true;
            } else {
                next_tma = start_single(t + stride);
            }
        }
        if (!run) {
            wait_box(next_tma);
            continue;
        }
        const double dt = ctl.dt;
        const double inv_h = 1.0 / gd.h;
        // ---- divergence, RK combination, stores ----------------------------
        double lmax = 0.0;
#pragma unroll
        for (int it = 0; it < CPT; ++it) {
            const int k = tid + it * NT;
            if (k >= TX * TY) break;
            const int r = k / TX, c = k - r * TX, i = tx0 + c, j = ty0 + r;
            if (i >= n || j >= n) continue;
            double res[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double *fx = FX + q * TY * (TX + 1) + r * (TX + 1) + c;
                const double *fy = FY + q * (TY + 1) * TX + r * TX + c;
                res[q] = -(fx[1] - fx[0]) * inv_h - (fy[TX] - fy[0]) * inv_h;
            }
            if (a.stage == 0) {
                double *rhs = (double *)a.rhs;
                const size_t n2 = (size_t)n * n, kk = (size_t)j * n + i;
                for (int q = 0; q < 4; ++q) rhs[q * n2 + kk] = res[q];
                ((double *)a.lam)[kk] = fabs(wk[it][1]) + fabs(wk[it][2]) +
                                        sound<double>(wk[it][3], wk[it][0], Gas<double>{gd.gam, gd.gam - 1.0});
                continue;
            }
            double w0[4], wq[4], c0[4], cv[4], w[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                wq[q] = wk[it][q];
                w0[q] = a.stage == 1 ? wk[it][q] : u0v[it][q];
            }
            c0[0] = w0[0]; c0[1] = w0[0] * w0[1]; c0[2] = w0[0] * w0[2];
            c0[3] = w0[3] * gf.igm1 + 0.5 * w0[0] * (w0[1] * w0[1] + w0[2] * w0[2]);
            if (a.stage == 1) {
#pragma unroll
                for (int q = 0; q < 4; ++q) cv[q] = c0[q] + dt * res[q];
            } else {
                double ck[4];
                ck[0] = wq[0]; ck[1] = wq[0] * wq[1]; ck[2] = wq[0] * wq[2];
                ck[3] = wq[3] * gf.igm1 + 0.5 * wq[0] * (wq[1] * wq[1] + wq[2] * wq[2]);
                if (a.stage == 2) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) cv[q] = 0.75 * c0[q] + 0.25 * (ck[q] + dt * res[q]);
                } else {
                    const double a3 = 1. / 3., b3 = 2. / 3.;
#pragma unroll
                    for (int q = 0; q < 4; ++q) cv[q] = a3 * c0[q] + b3 * (ck[q] + dt * res[q]);
                }
            }
            const double ir = frcp(cv[0]);
            w[0] = cv[0];
            w[1] = cv[1] * ir;
            w[2] = cv[2] * ir;
            w[3] = gf.gm1 * (cv[3] - 0.5 * (cv[1] * cv[1] + cv[2] * cv[2]) * ir);
            w[0] = floor14(w[0]);
            w[3] = floor14(w[3]);
            double *out = (double *)(a.stage == 1 ? gd.k1 : a.stage == 2 ? gd.k2 : gd.st[0]);
            put_cell<double>(gd, out, j, i, w);
            if (a.stage == 3) {
                const double lam = fabs(w[1]) + fabs(w[2]) + snd_rsq(gf.gam * w[3], w[0]);
                lmax = fmax(lmax, lam);
            }
        }
        // ---- max wave speed of the new state (stage 3) ---------------------
        if (a.stage == 3) {
            if (!batched && tid == 0 && tile == 0) leader_finish<P64>(gd.ctrl);
            if (batched) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
                if ((tid & 31) == 0 && lmax > 0.0)
                    atomicMax(&gd.ctrl->lam_acc, (unsigned long long)__double_as_longlong(lmax));
            } else {
                lacc = fmax(lacc, lmax);
            }
        }
        // ---- the next tile's box: wait, then release CE / FX / FY ----------
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
    if (s_err && gd_has_tma(a)) mbar_wait(&s_bar, phase);
}

// resident CTAs per SM a tile shape is compiled for: as many as the SM's
// 228 KB of shared memory holds (1 KB reserved per CTA, plus the static
// part), at most 24 warps, so a thread keeps >= 80 registers
template <int ORDER, int SHAPE>
struct Lean64K {
    static constexpr TileShape ts = kTileShapes[SHAPE];
    using LY = Lean64<ORDER, ts.tx, ts.ty>;
    static constexpr int kBySmem = (int)((228 * 1024) / (LY::kSmem + 1024 + 512));
    static constexpr int kByWarps = 768 / ts.nt;
    static constexpr int kMinBlocks = kBySmem < kByWarps ? kBySmem : kByWarps;
    static_assert(kMinBlocks >= 1, "one CTA fits");
};

template <int ORDER, int SHAPE, int RS>
static void *fn64(bool batched)
{
    using KK = Lean64K<ORDER, SHAPE>;
    constexpr TileShape ts = KK::ts;
    return batched ? (void *)stage64_kernel<ORDER, ts.tx, ts.ty, ts.nt, true, KK::kMinBlocks, RS>
                   : (void *)stage64_kernel<ORDER, ts.tx, ts.ty, ts.nt, false, KK::kMinBlocks, RS>;
}

template <int ORDER, int RS>
static void *fn64_shape(int shape, bool batched)
{
    switch (shape) {
    case 0: return fn64<ORDER, 0, RS>(batched);
    case 1: return fn64<ORDER, 1, RS>(batched);
    case 2: return fn64<ORDER, 2, RS>(batched);
    case 3: return fn64<ORDER, 3, RS>(batched);
    case 4: return fn64<ORDER, 4, RS>(batched);
    case 5: return fn64<ORDER, 5, RS>(batched);
    default: return nullptr;
    }
}

void *stage64_fn(int order, int shape, int rs, bool batched)
{
    if (order == 7 && rs == 0) return fn64_shape<7, 0>(shape, batched);
    return nullptr;
}

size_t stage64_smem(int order, int shape)
{
    if (shape < 0 || shape >= kNumTileShapes) return 0;
    const TileShape &ts = kTileShapes[shape];
    const int g = (order + 1) / 2;
    const size_t pl = (size_t)(ts.tx + 2 * g) * (ts.ty + 2 * g), cpl = (size_t)(ts.tx + 2) * (ts.ty + 2);
    return sizeof(double) * (4 * pl + 2 * cpl + 4 * ts.ty * (ts.tx + 1) + 4 * (ts.ty + 1) * ts.tx);
}

}  // namespace fvb
