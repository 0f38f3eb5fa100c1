// fvb_stage32c.cu -- the SSP-RK3 stage kernel of the FP32-compensated form.
//
// Same tile pipeline as the FP64 kernel (fvb_stage.cu): persistent CTAs walk
// the tiles of one grid or of a batch's tile table; the halo box of the next
// tile streams in through TMA while the current one is computed; every face
// is evaluated once; the RK combination stores the interior and its ghost
// images; stage 3 max-reduces the wave speed into the step control.
//
// What differs, for FP32 throughput: the faces are evaluated in pairs --
// x-face p in the low half and y-face p in the high half of packed FP32
// registers (fvb_face2.cuh) -- so the face arithmetic issues one instruction
// per two faces; and three CTAs of 256 threads share an SM (68 KB of shared
// memory and <= 85 registers each).
//
// State: conserved (rho, rho u, rho v, E) as an FP32 hi/lo pair per value;
// the stages form increments d1 = dt L(U0), d2 = (d1 + dt L(U1)) / 4 and add
// U = U0 + 2/3 (d2 + dt L(U2)) to the pair with an error-free sum, so the
// state keeps ~48 bits while all flux arithmetic is FP32.  Ping-pong state
// buffers (parity) keep U0 readable while U is written.
#include <stdint.h>

#include "fvb_internal.h"
#include "fvb_physics.cuh"
#include "fvb_device.cuh"
#include "fvb_tma.cuh"
#include "fvb_face2.cuh"

namespace fvb {

// resident CTAs per SM the kernel is compiled for: 768 threads (24 warps)
// per SM, <= 85 registers a thread
template <int NT> struct MinBlocks32c { static constexpr int v = 768 / NT; };

// The RK update of one cell from dres = dt L(U) (stage 1: d1 = dres; stage
// 2: d2 = (d1 + dres) / 4; stage 3: U0 + 2/3 (d2 + dres) added to the hi /
// lo pair with an error-free sum, floors, stores with ghost images, and the
// cell's wave speed into lmax).
__device__ __forceinline__ void update_cell32c(const GridDev &gd, int stage, int cur, int nxt, int j, int i,
                                               const float dres[4], float gam, float gm1, float &lmax)
{
    if (stage == 1) {
        put_cell<float>(gd, (float *)gd.k1, j, i, dres);
    } else if (stage == 2) {
        float d[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float d1 = ((const float *)gd.k1)[gidx(gd, q, j, i)];
            d[q] = 0.25f * (d1 + dres[q]);
        }
        put_cell<float>(gd, (float *)gd.k2, j, i, d);
    } else {
        float vh[4], vl[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const long long e = gidx(gd, q, j, i);
            const float d = (2.0f / 3.0f) * (((const float *)gd.k2)[e] + dres[q]);
            vh[q] = ((const float *)gd.st[cur])[e];
            vl[q] = ((const float *)gd.lo[cur])[e];
            df_add(vh[q], vl[q], d);
        }
        // floors rho, p >= 1e-14 on the new state
        float w[4];
        {
            const float ir = frcp(vh[0]);
            w[0] = vh[0]; w[1] = vh[1] * ir; w[2] = vh[2] * ir;
            w[3] = gm1 * (vh[3] - 0.5f * (vh[1] * vh[1] + vh[2] * vh[2]) * ir);
        }
        if (!(w[0] > 1e-14f)) { vh[0] = 1e-14f; vl[0] = 0.f; w[0] = 1e-14f; }
        if (!(w[3] > 1e-14f)) {
            float ke = 0.5f * (vh[1] * vh[1] + vh[2] * vh[2]) / vh[0];
            vh[3] = 1e-14f / gm1 + ke; vl[3] = 0.f; w[3] = 1e-14f;
        }
        put_cell2<float>(gd, (float *)gd.st[nxt], (float *)gd.lo[nxt], j, i, vh, vl);
        float cs2 = gam * w[3] * frcp(w[0]);
        float lam = fabsf(w[1]) + fabsf(w[2]) + fsqrt(cs2 > 1e-14f ? cs2 : 1e-14f);
        lmax = fmaxf(lmax, lam);  // (NaN skipped; exact in FP64 below)
    }
}

template <int TX, int TY, int NT, bool BATCHED>
__global__ void __launch_bounds__(NT, MinBlocks32c<NT>::v) stage32c_kernel(const __grid_constant__ StageArgs a)
{
    constexpr int G = 4;
    constexpr int SW = TX + 2 * G, SH = TY + 2 * G, PL = SW * SH;
    constexpr int NXF = (TX + 1) * TY, NYF = TX * (TY + 1);
    constexpr int NP = NXF > NYF ? NXF : NYF;
    constexpr int NC = TX * TY;
    constexpr int NW = NT / 32;

    // IN: the halo box as loaded (hi + increment planes); W: rho, u, v, p,
    // c, E the faces read; FX / FY: face fluxes
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float *IN = reinterpret_cast<float *>(smem_raw);
    float *W = IN + 8 * PL;
    float *FX = W + 6 * PL;               // [4][TY][TX+1]
    float *FY = FX + 4 * TY * (TX + 1);   // [4][TY+1][TX]
    __shared__ double s_red[NW];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ int s_err;
    __shared__ __align__(16) TileHdr s_hdr[2];
    __shared__ TileRef s_ref_next;  // batched: table entry of the CTA's next tile

    const int tid = threadIdx.x;
    constexpr bool batched = BATCHED;
    const int ntiles = batched ? *a.ntiles : a.ntiles_static;
    const int cur = a.parity, nxt = a.parity ^ 1;
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
    // The wait at the end of a tile needs no block barrier when the box came
    // through TMA: the next writes of every buffer are already ordered by
    // the barriers inside the tile (W by the conversion barrier, FX / FY by
    // the face barrier the update follows, IN by the conversion barrier the
    // next load is issued behind; the update reads neither W nor IN), and
    // each thread's own wait makes the box visible to it.  A box loaded by
    // the threads themselves needs the barrier.  A timeout is agreed on at
    // the next conversion barrier.
    auto wait_box_own = [&](bool tma) {
        if (tma) {
            if (mbar_wait(&s_bar, phase)) phase ^= 1;
            else s_err = 1;
        } else {
            __syncthreads();
        }
    };
    // single grid: start the halo-box load of tile t (every thread: the
    // plain path loads cooperatively)
    auto start_single = [&](int t) -> bool {
        if (tid == 0 && a.grid.tmap) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue_tile_load<P32C, G, SW, SH, NT>(a.grid, a.stage, cur, t, IN, &s_bar, tid);
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
            start_batched_tile<P32C, G, SW, SH, NT>(a, &s_hdr[0], r0, hdr_word(a, r0, tid), cur, IN, &s_bar, tid);
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
    // which of this thread's conversion cells (k = tid + it NT) the HLLE
    // reads the sound speed and energy of: the interior rows x columns
    // [G-1, G+TX], and rows G-1, G+TY x the interior columns
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
    // one grid: the step control is the same for every tile of the launch,
    // read once (the leader is CTA 0, whose first tile is tile 0)
    TileCtl ctl1{};
    if (!batched && t < ntiles) ctl1 = tile_control<P32C>(a.grid.ctrl, a.stage, tid == 0 && t == 0);
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
        const float gam = (float)gd.gam, gm1 = (float)gd.gam - 1.0f, igm1 = (float)(1.0 / (gd.gam - 1.0));
        // ---- 1. stage input U0 + d into W as primitives (+ c, E where the
        //         HLLE reads them, cemask) ------------------------------------
        if (ctl.run) {
#pragma unroll
            for (int it = 0; it < NCV; ++it) {
                const int k = tid + it * NT;
                if (k >= PL) break;
                float w0 = IN[k], w1 = IN[PL + k], w2 = IN[2 * PL + k], w3 = IN[3 * PL + k];
                if (a.stage >= 2) {
                    w0 += IN[4 * PL + k]; w1 += IN[5 * PL + k]; w2 += IN[6 * PL + k]; w3 += IN[7 * PL + k];
                }
                const bool ce = (cemask >> it) & 1u;
                const float ir = frcp(w0);
                const float E = w3;
                w1 *= ir;
                w2 *= ir;
                w3 = gm1 * (E - 0.5f * w0 * (w1 * w1 + w2 * w2));
                if (ce) {
                    const float cs2 = gam * w3 * ir;
                    W[4 * PL + k] = fsqrt(cs2 > 1e-14f ? cs2 : 1e-14f);
                    W[5 * PL + k] = E;
                }
                W[k] = w0; W[PL + k] = w1; W[2 * PL + k] = w2; W[3 * PL + k] = w3;
            }
        }
        __syncthreads();
        // a halo load that never arrived (seen by any thread): record it and
        // stop; every thread reads s_err after the same barrier
        if (s_err) {
            if (tid == 0 && gd.ctrl) gd.ctrl->status = FVB_ERR_TIMEOUT;
            break;
        }
        // ---- 2. load the next tile into IN (asynchronous through TMA) -------
        // (in a batched launch warp 0 also fetches that tile's header)
        bool next_tma = false;
        if (has_next) {
            if (batched) {
                if (tid < 32) {
                    start_batched_tile<P32C, G, SW, SH, NT>(a, &s_hdr[slot ^ 1], ref_next, wnext, cur, IN, &s_bar,
                                                            tid);
                    if (tid == 0) s_ref_next = ref_after;
                }
                next_tma = true;
            } else {
                next_tma = start_single(t + stride);
            }
        }
        if (!ctl.run) {
            if (ctl.copy) {
                // skipped step: the next step reads the other buffer
                const float *hi = (const float *)gd.st[cur], *lo = (const float *)gd.lo[cur];
                for (int k = tid; k < NC; k += NT) {
                    int r = k / TX, c = k - r * TX, i = tx0 + c, j = ty0 + r;
                    if (i >= n || j >= n) continue;
                    float vh[4], vl[4];
                    long long e = gidx(gd, 0, j, i);
                    for (int q = 0; q < 4; ++q) { vh[q] = hi[e + q * gd.plane]; vl[q] = lo[e + q * gd.plane]; }
                    put_cell2<float>(gd, (float *)gd.st[nxt], (float *)gd.lo[nxt], j, i, vh, vl);
                }
            }
            wait_box(next_tma);
            continue;
        }
        const float dt = (float)ctl.dt;
        const float dt_h = dt * (float)(1.0 / gd.h);

        // ---- 3. face fluxes, x-face p and y-face p as one packed pair -------
        for (int p = tid; p < NP; p += NT) {
            const int px = p < NXF ? p : NXF - 1, py = p < NYF ? p : NYF - 1;
            const int rx = px / (TX + 1), cx = px - rx * (TX + 1);
            const int ry = py / TX, cy = py - ry * TX;
            const int bx = (rx + G) * SW + (cx + G), by = (ry + G) * SW + (cy + G);
            f2::V L[4], Rv[4], WL[4], WR[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                // x lane: (rho, u, v, p) along x; y lane: (rho, v, u, p) along y
                const float *vx = W + m * PL + bx;
                const float *vy = W + (m == 1 ? 2 : m == 2 ? 1 : m) * PL + by;
                f2::V s[8];
#pragma unroll
                for (int d = 0; d < 8; ++d) s[d] = make_float2(vx[d - G], vy[(d - G) * SW]);
                f2::upface7(s, L[m], Rv[m]);
                WL[m] = s[G - 1];
                WR[m] = s[G];
            }
            const f2::V tiny = f2::splat(1e-14f);
            L[0] = f2::vmax(L[0], tiny); Rv[0] = f2::vmax(Rv[0], tiny);
            L[3] = f2::vmax(L[3], tiny); Rv[3] = f2::vmax(Rv[3], tiny);
            const float *cex = W + 4 * PL + bx, *cey = W + 4 * PL + by;
            f2::V F[4];
            f2::face_flux(L, Rv, WL, WR, make_float2(cex[-1], cey[-SW]), make_float2(cex[0], cey[0]),
                          make_float2(cex[PL - 1], cey[PL - SW]), make_float2(cex[PL], cey[PL]), gam, igm1, F);
            if (p < NXF) {
                float *o = FX + rx * (TX + 1) + cx;
                constexpr int os = TY * (TX + 1);
                o[0] = F[0].x; o[os] = F[1].x; o[2 * os] = F[2].x; o[3 * os] = F[3].x;
            }
            if (p < NYF) {
                float *o = FY + ry * TX + cy;
                constexpr int os = (TY + 1) * TX;
                // y lane: normal momentum is v, tangential u
                o[0] = F[0].y; o[os] = F[2].y; o[2 * os] = F[1].y; o[3 * os] = F[3].y;
            }
        }
        __syncthreads();

        // ---- 4. divergence, RK combination, stores --------------------------
        float lmax = 0.0f;
        for (int k = tid; k < NC; k += NT) {
            const int r = k / TX, c = k - r * TX, i = tx0 + c, j = ty0 + r;
            if (i >= n || j >= n) continue;
            float dres[4];  // dt L
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float *fx = FX + q * TY * (TX + 1) + r * (TX + 1) + c;
                const float *fy = FY + q * (TY + 1) * TX + r * TX + c;
                dres[q] = -((fx[1] - fx[0]) + (fy[TX] - fy[0])) * dt_h;
            }
            update_cell32c(gd, a.stage, cur, nxt, j, i, dres, gam, gm1, lmax);
        }

        // ---- 5. max wave speed of the new state (stage 3) ------------------
        if (a.stage == 3) {
            // (a batched launch advances each grid's time where its tile 0's header is published)
            if (!batched && tid == 0 && tile == 0) leader_finish<P32C>(gd.ctrl);
            if (batched) {
                // tiles of one CTA belong to different grids: one atomic per
                // warp and tile
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
                if ((tid & 31) == 0 && lmax > 0.0f)
                    atomicMax(&gd.ctrl->lam_acc, (unsigned long long)__double_as_longlong((double)lmax));
            } else {
                lacc = fmax(lacc, (double)lmax);
            }
        }
        // ---- 6. next tile's halo box -----------------------------------------
        wait_box_own(next_tma);
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
// Row-pair variant of the compensated stage kernel (tile variant 6).
//
// The two lanes of every packed register are the same face, or the same
// cell, in two rows HT = TY / 2 apart: the working tile keeps each quantity
// as float2 pairs (box row r', box row r' + HT) for r' in [0, HT + 2G), so
// one 64-bit shared load fetches a stencil point for both faces, x-faces
// pair with x-faces and y-faces with y-faces (the same index pattern and
// component order in both lanes), and the face fluxes are stored and read
// back as pairs.  The halo box, the tile walk, the step control and the
// per-cell update are those of stage32c_kernel above; the rows the two
// halves share (box rows HT .. 2G + HT - 1) are converted once per half.
// ---------------------------------------------------------------------------
template <int TX, int TY>
struct RowPair {
    static constexpr int G = 4, HT = TY / 2;
    static constexpr int SW = TX + 2 * G, SH = TY + 2 * G, PL = SW * SH;
    static constexpr int PR = HT + 2 * G;             // pair rows of the working tile
    static constexpr int P2 = PR * SW;                // pairs per working plane
    static constexpr int C2 = (HT + 2) * SW;          // pairs of the c / E planes: rows G-1 .. G+HT
    static constexpr int NXP = HT * (TX + 1);         // x-face pairs
    static constexpr int NYP = (HT + 1) * TX;         // y-face pairs (row HT is evaluated in both halves)
    static constexpr int NC2 = HT * TX;               // cell pairs
    static constexpr size_t smem = sizeof(float) * 8 * PL +
                                   sizeof(float2) * (4 * P2 + 2 * C2 + 4 * HT * (TX + 1) + 4 * (HT + 1) * TX);
};

template <int TX, int TY, int NT, bool BATCHED>
__global__ void __launch_bounds__(NT, MinBlocks32c<NT>::v) stage32p_kernel(const __grid_constant__ StageArgs a)
{
    using RP = RowPair<TX, TY>;
    static_assert(TY % 2 == 0, "two halves of equal height");
    constexpr int G = RP::G, HT = RP::HT, SW = RP::SW, SH = RP::SH, PL = RP::PL;
    constexpr int P2 = RP::P2, C2 = RP::C2, NXP = RP::NXP, NYP = RP::NYP, NC2 = RP::NC2;
    constexpr int NC = TX * TY;
    constexpr int NW = NT / 32;
    constexpr int HS = HT * SW;  // box offset of the upper half's rows

    // IN: the halo box as loaded (hi + increment planes); W2: rho, u, v, p
    // as row pairs; CE2: sound speed and energy as row pairs (pair rows G-1
    // .. G+HT); FX2 / FY2: face fluxes as row pairs
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float *IN = reinterpret_cast<float *>(smem_raw);
    float2 *W2 = reinterpret_cast<float2 *>(IN + 8 * PL);
    float2 *CE2 = W2 + 4 * P2;
    float2 *FX2 = CE2 + 2 * C2;              // [4][HT][TX+1]
    float2 *FY2 = FX2 + 4 * HT * (TX + 1);   // [4][HT+1][TX]
    __shared__ double s_red[NW];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ int s_err;
    __shared__ __align__(16) TileHdr s_hdr[2];
    __shared__ TileRef s_ref_next;

    const int tid = threadIdx.x;
    constexpr bool batched = BATCHED;
    const int ntiles = batched ? *a.ntiles : a.ntiles_static;
    const int cur = a.parity, nxt = a.parity ^ 1;
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
    // end-of-tile wait without a block barrier for a TMA-fed box, as in
    // stage32c_kernel (W2 / FX2 / FY2 in place of W / FX / FY)
    auto wait_box_own = [&](bool tma) {
        if (tma) {
            if (mbar_wait(&s_bar, phase)) phase ^= 1;
            else s_err = 1;
        } else {
            __syncthreads();
        }
    };
    auto start_single = [&](int t) -> bool {
        if (tid == 0 && a.grid.tmap) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue_tile_load<P32C, G, SW, SH, NT>(a.grid, a.stage, cur, t, IN, &s_bar, tid);
        return a.grid.tmap != nullptr;
    };
    // failure injection (fvb_debug_drop_load), as in stage32c_kernel
    const bool drop = !batched && blockIdx.x == 0 && a.stage > 0 && a.grid.ctrl && a.grid.tmap &&
                      *(volatile int *)&a.grid.ctrl->drop_load;
    const int stride = gridDim.x;
    int t = blockIdx.x, slot = 0;
    if (t < ntiles && batched) {
        if (tid < 32) {
            const TileRef r0 = a.tiles[t];
            start_batched_tile<P32C, G, SW, SH, NT>(a, &s_hdr[0], r0, hdr_word(a, r0, tid), cur, IN, &s_bar, tid);
            if (tid == 0 && t + stride < ntiles) s_ref_next = a.tiles[t + stride];
        }
        wait_box(true);
    } else if (drop) {
        wait_box(true);
        if (tid == 0) a.grid.ctrl->drop_load = 0;
    } else {
        wait_box(t < ntiles ? start_single(t) : false);
    }
    double lacc = 0.0;
    // which of this thread's conversion pairs (k = tid + it NT) the HLLE reads
    // the sound speed and energy of: pair rows G-1 .. G+HT, columns G-1 .. G+TX
    constexpr int NCV = (P2 + NT - 1) / NT;
    static_assert(NCV <= 32, "one mask bit per conversion pair");
    unsigned cemask = 0;
#pragma unroll
    for (int it = 0; it < NCV; ++it) {
        const int k = tid + it * NT, r = k / SW, c = k - r * SW;
        const bool ce = (unsigned)(r - (G - 1)) < (unsigned)(HT + 2) && (unsigned)(c - (G - 1)) < (unsigned)(TX + 2);
        cemask |= (ce && k < P2 ? 1u : 0u) << it;
    }
    TileCtl ctl1{};
    if (!batched && t < ntiles) ctl1 = tile_control<P32C>(a.grid.ctrl, a.stage, tid == 0 && t == 0);
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
        const float gam = (float)gd.gam, gm1 = (float)gd.gam - 1.0f, igm1 = (float)(1.0 / (gd.gam - 1.0));
        // ---- 1. stage input U0 + d into W2 as primitive row pairs (+ c, E
        //         where the HLLE reads them) -----------------------------------
        if (ctl.run) {
            const f2::V nhalf = f2::splat(-0.5f), G1 = f2::splat(gm1), GA = f2::splat(gam);
#pragma unroll
            for (int it = 0; it < NCV; ++it) {
                const int k = tid + it * NT;
                if (k >= P2) break;
                f2::V w0 = make_float2(IN[k], IN[k + HS]), w1 = make_float2(IN[PL + k], IN[PL + k + HS]);
                f2::V w2 = make_float2(IN[2 * PL + k], IN[2 * PL + k + HS]);
                f2::V w3 = make_float2(IN[3 * PL + k], IN[3 * PL + k + HS]);
                if (a.stage >= 2) {
                    w0 = f2::add(w0, make_float2(IN[4 * PL + k], IN[4 * PL + k + HS]));
                    w1 = f2::add(w1, make_float2(IN[5 * PL + k], IN[5 * PL + k + HS]));
                    w2 = f2::add(w2, make_float2(IN[6 * PL + k], IN[6 * PL + k + HS]));
                    w3 = f2::add(w3, make_float2(IN[7 * PL + k], IN[7 * PL + k + HS]));
                }
                const f2::V ir = f2::rcp(w0);
                const f2::V E = w3;
                w1 = f2::mul(w1, ir);
                w2 = f2::mul(w2, ir);
                // p = (gamma - 1)(E - rho (u^2 + v^2) / 2)
                w3 = f2::mul(G1, f2::fma(f2::mul(nhalf, w0), f2::fma(w1, w1, f2::mul(w2, w2)), E));
                if ((cemask >> it) & 1u) {
                    const f2::V cs2 = f2::mul(f2::mul(GA, w3), ir);
                    const int kc = k - (G - 1) * SW;
                    CE2[kc] = f2::vsqrt(f2::vmax(cs2, f2::splat(1e-14f)));
                    CE2[C2 + kc] = E;
                }
                W2[k] = w0; W2[P2 + k] = w1; W2[2 * P2 + k] = w2; W2[3 * P2 + k] = w3;
            }
        }
        __syncthreads();
        // a halo load that never arrived (seen by any thread): record it and
        // stop; every thread reads s_err after the same barrier
        if (s_err) {
            if (tid == 0 && gd.ctrl) gd.ctrl->status = FVB_ERR_TIMEOUT;
            break;
        }
        // ---- 2. load the next tile into IN (asynchronous through TMA) -------
        bool next_tma = false;
        if (has_next) {
            if (batched) {
                if (tid < 32) {
                    start_batched_tile<P32C, G, SW, SH, NT>(a, &s_hdr[slot ^ 1], ref_next, wnext, cur, IN, &s_bar,
                                                            tid);
                    if (tid == 0) s_ref_next = ref_after;
                }
                next_tma = true;
            } else {
                next_tma = start_single(t + stride);
            }
        }
        if (!ctl.run) {
            if (ctl.copy) {
                // skipped step: the next step reads the other buffer
                const float *hi = (const float *)gd.st[cur], *lo = (const float *)gd.lo[cur];
                for (int k = tid; k < NC; k += NT) {
                    int r = k / TX, c = k - r * TX, i = tx0 + c, j = ty0 + r;
                    if (i >= n || j >= n) continue;
                    float vh[4], vl[4];
                    long long e = gidx(gd, 0, j, i);
                    for (int q = 0; q < 4; ++q) { vh[q] = hi[e + q * gd.plane]; vl[q] = lo[e + q * gd.plane]; }
                    put_cell2<float>(gd, (float *)gd.st[nxt], (float *)gd.lo[nxt], j, i, vh, vl);
                }
            }
            wait_box(next_tma);
            continue;
        }
        const float dt = (float)ctl.dt;
        const float dt_h = dt * (float)(1.0 / gd.h);

        // ---- 3. face fluxes as row pairs: x-faces, then y-faces -------------
        const f2::V tiny = f2::splat(1e-14f);
        for (int p = tid; p < NXP; p += NT) {
            // x-faces of rows r and r + HT at column c (the face left of cell c)
            const int r = p / (TX + 1), c = p - r * (TX + 1);
            const int base = (r + G) * SW + (c + G);
            f2::V L[4], Rv[4], WL[4], WR[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const f2::V *v = W2 + m * P2 + base;
                f2::V s[8];
#pragma unroll
                for (int d = 0; d < 8; ++d) s[d] = v[d - G];
                f2::upface7(s, L[m], Rv[m]);
                WL[m] = s[G - 1];
                WR[m] = s[G];
            }
            L[0] = f2::vmax(L[0], tiny); Rv[0] = f2::vmax(Rv[0], tiny);
            L[3] = f2::vmax(L[3], tiny); Rv[3] = f2::vmax(Rv[3], tiny);
            const f2::V *ce = CE2 + (r + 1) * SW + (c + G - 1);
            f2::V F[4];
            f2::face_flux(L, Rv, WL, WR, ce[0], ce[1], ce[C2], ce[C2 + 1], gam, igm1, F);
            f2::V *o = FX2 + p;
            constexpr int os = HT * (TX + 1);
            o[0] = F[0]; o[os] = F[1]; o[2 * os] = F[2]; o[3 * os] = F[3];
        }
        for (int p = tid; p < NYP; p += NT) {
            // y-faces of rows r and r + HT (below cell rows r, r + HT) at column c
            const int r = p / TX, c = p - r * TX;
            const int base = (r + G) * SW + (c + G);
            f2::V L[4], Rv[4], WL[4], WR[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                // (rho, v, u, p): normal velocity v, tangential u
                const f2::V *v = W2 + (m == 1 ? 2 : m == 2 ? 1 : m) * P2 + base;
                f2::V s[8];
#pragma unroll
                for (int d = 0; d < 8; ++d) s[d] = v[(d - G) * SW];
                f2::upface7(s, L[m], Rv[m]);
                WL[m] = s[G - 1];
                WR[m] = s[G];
            }
            L[0] = f2::vmax(L[0], tiny); Rv[0] = f2::vmax(Rv[0], tiny);
            L[3] = f2::vmax(L[3], tiny); Rv[3] = f2::vmax(Rv[3], tiny);
            const f2::V *ce = CE2 + r * SW + (c + G);
            f2::V F[4];
            f2::face_flux(L, Rv, WL, WR, ce[0], ce[SW], ce[C2], ce[C2 + SW], gam, igm1, F);
            f2::V *o = FY2 + p;
            constexpr int os = (HT + 1) * TX;
            // normal momentum is v, tangential u
            o[0] = F[0]; o[os] = F[2]; o[2 * os] = F[1]; o[3 * os] = F[3];
        }
        __syncthreads();

        // ---- 4. divergence as pairs, then each cell's RK update -------------
        float lmax = 0.0f;
        const f2::V ndt = f2::splat(-dt_h);
        for (int cp = tid; cp < NC2; cp += NT) {
            const int r = cp / TX, c = cp - r * TX, i = tx0 + c;
            f2::V dr[4];  // dt L of cells (r, c) and (r + HT, c)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const f2::V *fx = FX2 + q * HT * (TX + 1) + r * (TX + 1) + c;
                const f2::V *fy = FY2 + q * (HT + 1) * TX + r * TX + c;
                dr[q] = f2::mul(f2::add(f2::sub(fx[1], fx[0]), f2::sub(fy[TX], fy[0])), ndt);
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int j = ty0 + r + h * HT;
                if (i >= n || j >= n) continue;
                float dres[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) dres[q] = h ? dr[q].y : dr[q].x;
                update_cell32c(gd, a.stage, cur, nxt, j, i, dres, gam, gm1, lmax);
            }
        }

        // ---- 5. max wave speed of the new state (stage 3) ------------------
        if (a.stage == 3) {
            if (!batched && tid == 0 && tile == 0) leader_finish<P32C>(gd.ctrl);
            if (batched) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
                if ((tid & 31) == 0 && lmax > 0.0f)
                    atomicMax(&gd.ctrl->lam_acc, (unsigned long long)__double_as_longlong((double)lmax));
            } else {
                lacc = fmax(lacc, (double)lmax);
            }
        }
        // ---- 6. next tile's halo box -----------------------------------------
        wait_box_own(next_tma);
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

template <int SHAPE>
static void *fn32c(bool batched)
{
    constexpr TileShape ts = kTileShapes[SHAPE];
    if constexpr (SHAPE == kRowPairShape)
        return batched ? (void *)stage32p_kernel<ts.tx, ts.ty, ts.nt, true>
                       : (void *)stage32p_kernel<ts.tx, ts.ty, ts.nt, false>;
    else
        return batched ? (void *)stage32c_kernel<ts.tx, ts.ty, ts.nt, true>
                       : (void *)stage32c_kernel<ts.tx, ts.ty, ts.nt, false>;
}

void *stage32c_fn(int shape, bool batched)
{
    switch (shape) {
    case 0: return fn32c<0>(batched);
    case 1: return fn32c<1>(batched);
    case 2: return fn32c<2>(batched);
    case 3: return fn32c<3>(batched);
    case 4: return fn32c<4>(batched);
    case 5: return fn32c<5>(batched);
    case 6: return fn32c<6>(batched);
    default: return nullptr;
    }
}

size_t stage32c_smem(int shape)
{
    if (shape < 0 || shape >= kNumTileShapes) return 0;
    if (shape == kRowPairShape)
        return RowPair<kTileShapes[kRowPairShape].tx, kTileShapes[kRowPairShape].ty>::smem;
    const TileShape &ts = kTileShapes[shape];
    const int sw = ts.tx + 8, sh = ts.ty + 8;
    return sizeof(float) * ((size_t)14 * sw * sh + 4 * ts.ty * (ts.tx + 1) + 4 * (ts.ty + 1) * ts.tx);
}

}  // namespace fvb
