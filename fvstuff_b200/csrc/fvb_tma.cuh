// fvb_tma.cuh -- TMA halo-box loads and bounded mbarrier waits shared by
// the stage kernels (no cluster multicast anywhere), and the tile headers of
// batched launches.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include "fvb_internal.h"
#include "fvb_device.cuh"

namespace fvb {

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// plain arrival (no transaction bytes): completes the phase of a barrier
// initialised with count 1
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// one 3-D tiled tensor load global -> shared, completing on `bar`
__device__ __forceinline__ void tma_load3(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// bounded wait for phase `parity` of `bar`: false once one second of GPU
// time (%globaltimer) has passed without the phase completing
__device__ __forceinline__ uint64_t gtimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    constexpr uint64_t kLimitNs = 1000000000ull;
    uint64_t t0 = 0;
    for (uint32_t it = 0;; ++it) {
        uint32_t ok;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if ((it & 63) == 0) {
            const uint64_t now = gtimer_ns();
            if (it == 0) t0 = now;
            else if (now - t0 > kLimitNs) return false;
        }
    }
}

// The halo box of a tile in one grid: TMA when the grid has descriptors,
// else cooperative loads by the whole CTA (the caller's IDX_P arrays).
template <int PREC, int G, int SW, int SH, int NT, class R>
__device__ __forceinline__ void issue_tile_load(const GridDev &gd, int stage, int parity, int tile, R *IN,
                                                uint64_t *bar, int tid)
{
    constexpr int TXd = SW - 2 * G, TYd = SH - 2 * G;
    const int tx0 = (tile % gd.tiles_x) * TXd, ty0 = (tile / gd.tiles_x) * TYd;
    const bool two = (PREC == P32C) && (stage == 2 || stage == 3);
    if (gd.tmap) {
        if (tid == 0) {
            constexpr uint32_t box = 4u * SW * SH * sizeof(R);
            mbar_expect_tx(bar, two ? 2 * box : box);
            int m0;
            if (PREC == P32C) m0 = parity ? TM_ST1 : TM_ST0;
            else m0 = stage == 2 ? TM_K1 : stage == 3 ? TM_K2 : TM_ST0;
            const int x = gd.xoff + tx0;
            tma_load3(IN, gd.tmap + m0, x, ty0, 0, bar);
            if (two) tma_load3(IN + 4 * SW * SH, gd.tmap + (stage == 2 ? TM_K1 : TM_K2), x, ty0, 0, bar);
        }
        return;
    }
    const R *src = (const R *)(PREC == P32C ? gd.st[parity]
                                            : (stage == 2 ? gd.k1 : stage == 3 ? gd.k2 : gd.st[0]));
    const R *inc = two ? (const R *)(stage == 2 ? gd.k1 : gd.k2) : nullptr;
    const int np = gd.n + 2 * G;
    for (int k = tid; k < SH * SW; k += NT) {
        int r = k / SW, c = k - r * SW;
        int jp = ty0 + r, ip = tx0 + c;
        bool in = jp < np && ip < np;
        long long e = (long long)jp * gd.pitch + ip + gd.xoff;
        for (int q = 0; q < 4; ++q) {
            IN[q * SH * SW + k] = in ? src[e + q * gd.plane] : R(0);
            if (two) IN[(4 + q) * SH * SW + k] = in ? inc[e + q * gd.plane] : R(0);
        }
    }
}

// Tile headers of a batched launch.  Warp 0 stages them one tile ahead:
// the table entry of the CTA's next tile is loaded a tile early, and at the
// top of each tile each lane of warp 0 loads one 8-byte word of the next
// tile's grid descriptor or of its grid's step control (Ctrl), so these
// loads are in flight while the tile is converted.  After the conversion
// barrier warp 0 stores the words into shared memory, lane 0 evaluates the
// stage's step control of that grid from the copy (the lane that publishes a
// grid's tile 0 is that grid's leader and makes the stage's control writes,
// including the time advance of stage 3) and starts the next halo-box load;
// every thread reads the header after the barrier that ends the tile.  So a
// batched stage needs no separate step-control launch.  (A single-grid
// launch reads its grid from the kernel parameter and evaluates the step
// control once: it is the same for every tile.)
struct TileHdr {
    GridDev gd;
    Ctrl c;
    TileCtl ctl;
    int tile;
    int pad;
};
constexpr int kGridWords = (int)(sizeof(GridDev) / 8);
constexpr int kHdrWords = kGridWords + (int)(sizeof(Ctrl) / 8);
static_assert(sizeof(GridDev) % 8 == 0 && sizeof(Ctrl) % 8 == 0 && kHdrWords <= 32, "one warp copies a header");
static_assert(offsetof(TileHdr, c) == sizeof(GridDev), "grid descriptor and step control are contiguous");

// the grid of the current tile: its header in shared memory (batched) or
// the kernel parameter (single grid); a reference, so each field is read
// where it is used rather than held in registers across the tile
template <bool BATCHED>
__device__ __forceinline__ const GridDev &tile_grid(const TileHdr &h, const StageArgs &a)
{
    if constexpr (BATCHED) return h.gd;
    else return a.grid;
}

__device__ __forceinline__ unsigned long long hdr_word(const StageArgs &a, TileRef r, int lane)
{
    if (lane < kGridWords) return reinterpret_cast<const unsigned long long *>(a.grids + r.grid)[lane];
    if (lane < kHdrWords) return reinterpret_cast<const unsigned long long *>(a.ctrls + r.grid)[lane - kGridWords];
    return 0ull;
}

// warp 0: publish the header of tile r into h, evaluate its grid's step
// control for this stage, and start its halo-box load
template <int PREC, int G, int SW, int SH, int NT, class R>
__device__ __forceinline__ void start_batched_tile(const StageArgs &a, TileHdr *h, TileRef r, unsigned long long w,
                                                   int parity, R *IN, uint64_t *bar, int lane)
{
    if (lane < kHdrWords) reinterpret_cast<unsigned long long *>(h)[lane] = w;
    __syncwarp();
    if (lane == 0) {
        h->tile = r.tile;
        Ctrl *ctrl = a.ctrls + r.grid;
        const bool leader = r.tile == 0;
        h->ctl = step_control<PREC>(h->c, ctrl, a.stage, leader);
        if (a.stage == 3 && leader && h->ctl.run) leader_finish_from<PREC>(h->c, ctrl);
        if (h->gd.tmap) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue_tile_load<PREC, G, SW, SH, NT>(h->gd, a.stage, parity, r.tile, IN, bar, 0);
        } else {
            // batched grids load through TMA only: never compute on a box
            // that was not loaded
            mbar_arrive(bar);
            h->ctl.run = 0;
            h->ctl.copy = 0;
            if (r.tile == 0) ctrl->status = FVB_ERR_INVALID;
        }
    }
    __syncwarp();
}

}  // namespace fvb
