// fvb_internal.h -- device-side data structures shared by the kernels and
// the host library.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/fvb.h"

namespace fvb {

// Device-resident step control of one grid.  The stage kernels read and
// update it themselves, so a run of steps needs no host round trip:
//   stage 1 : every CTA derives dt from lam_acc (max wave speed of the
//             current state), t and t_stop, identically; the CTA holding
//             tile 0 ("leader") publishes dt / active
//   stage 2 : leader clears lam_acc
//   stage 3 : every CTA max-reduces lam of the new state into lam_acc;
//             leader advances t and step
// Fields a stage writes are never read by another CTA of the same stage.
struct Ctrl {
    double t;                   // simulated time (always FP64)
    double t_stop;              // steps stop when t >= t_stop
    double dt;                  // dt of the step in progress
    double cfl, h;              // dt = cfl * h / lam
    unsigned long long lam_acc; // bit pattern of max lam (non-negative double)
    unsigned long long lam_cur; // lam_acc that set the current dt
    long long step;
    int active;                 // the step in progress runs
    int status;                 // fvb_status of the step control
    int clamped;                // dt was clamped to land on t_stop
    int drop_load;              // failure-injection hook: the next single-grid stage launch
                                // issues no first halo-box load (its wait must run out)
    unsigned long long aux;     // KEEP: bit pattern of the entropy-distance max of the stage
                                // input; rec3: count of 2x2 blocks given the brutal mean fix
};

// Device view of one grid.  Element (q, jp, ip) of a padded buffer, padded
// coordinates jp, ip in [0, n + 2g), sits at q*plane + jp*pitch + xoff + ip.
// The IDX_P layout of the reference is pitch = n + 2g, xoff = 0,
// plane = pitch * (n + 2g).
struct GridDev {
    int n, g;
    int pitch, xoff;
    long long plane;
    int bcx, bcy;
    double h, gam;
    void *st[2];    // state: prim (F64/F32, st[0] only) or conserved hi (F32C, ping-pong)
    void *lo[2];    // F32C: lo words of the conserved state
    void *k1, *k2;  // stage outputs: U1/U2 primitives (F64/F32) or increments d1/d2 (F32C)
    Ctrl *ctrl;
    const CUtensorMap *tmap;  // TMA descriptors of st[0], st[1], k1, k2 for the
                              // kernel's halo box (device memory); null: plain loads
    int tiles_x;    // tiles along x for the kernel's tile width
    int pad;
};

enum { TM_ST0 = 0, TM_ST1 = 1, TM_K1 = 2, TM_K2 = 3, TM_COUNT = 4 };

// Tile-table entry of the batched launch: grid index and tile index.
struct TileRef {
    int grid;
    int tile;
};

enum Prec { P64 = 0, P32 = 1, P32C = 2 };

// Step control of one grid for one RK stage: the dt the stage uses, whether
// its tiles compute, and (FP32c stage 3 of a grid that stopped) whether they
// carry the state to the other buffer.
struct TileCtl {
    double dt;
    int run;
    int copy;
};

struct StageArgs {
    GridDev grid;              // single-grid launches
    const GridDev *grids;      // batched launches: grid descriptors
    Ctrl *ctrls;               // batched launches: step control of each grid (indexed like grids)
    const TileRef *tiles;      // batched launches: tile table
    const int *ntiles;         // batched launches: live tile count (device)
    int ntiles_static;         // single-grid launches: tiles
    int stage;                 // 1, 2, 3; 0 = residual only (reference contract)
    int parity;                // F32C: index of the current state buffer
    void *rhs, *lam;           // stage 0 outputs, (4, n, n) and (n, n) unpadded
};

// Tile shapes the stage kernel is instantiated for (tile width x height,
// threads per CTA).  Chosen so the face count (TX+1)TY + TX(TY+1) is close
// to a multiple of the thread count.
struct TileShape {
    int tx, ty, nt;
};
constexpr int kNumTileShapes = 7;
constexpr TileShape kTileShapes[kNumTileShapes] = {
    {32, 15, 256}, {32, 7, 128}, {64, 7, 256}, {16, 15, 256}, {32, 9, 256}, {32, 16, 256}, {32, 14, 256}};
// the variant whose FP32-compensated kernel evaluates faces and cells as
// pairs of rows TY/2 apart (fvb_stage32c.cu, stage32p_kernel); the FP64 and
// FP32 kernels treat it as one more tile shape
constexpr int kRowPairShape = 6;

// TMA descriptors (fvb_stage.cu): encode the four maps of a grid for a
// tile shape into host memory; false if this grid cannot use TMA
bool encode_tile_maps(const GridDev &gd, int prec, int order, int shape, CUtensorMap out[TM_COUNT]);
// stream-ordered copy of encoded maps into device memory (dst 64-byte aligned)
cudaError_t put_tile_maps(const CUtensorMap maps[TM_COUNT], CUtensorMap *dst, cudaStream_t s);

// the FP32-compensated stage kernel of a tile shape and its shared memory
// (fvb_stage32c.cu)
void *stage32c_fn(int shape, bool batched);
size_t stage32c_smem(int shape);

// launchers (fvb_stage.cu).  rs: the solver on the reconstructed states of
// the FP64 UP7 kernel -- 0 HLLC, 1 HLL, 2 Roe
cudaError_t launch_stage(int prec, int order, int shape, const StageArgs &a, int grid_ctas,
                         cudaStream_t s, int rs = 0);
size_t stage_smem_bytes(int prec, int order, int shape, int rs = 0);
int stage_max_ctas_per_sm(int prec, int order, int shape, int rs = 0);

// What a persistent launch of kernel `fn` with `threads` threads and `smem`
// bytes of dynamic shared memory needs on the current device: the shared-
// memory opt-in is applied and the resident CTAs per SM and the SM count
// are read once per (kernel, device, threads, smem), under a lock, so
// solvers on several host threads or devices set it up safely
// (fvb_stage.cu).  An error if not even one CTA fits on an SM.
struct LaunchFacts {
    int ctas_per_sm;
    int sms;
};
cudaError_t launch_facts(const void *fn, int threads, size_t smem, LaunchFacts &out);

}  // namespace fvb
