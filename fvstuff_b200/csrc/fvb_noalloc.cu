// fvb_noalloc.cu -- SSP-RK3 steps of a caller-held FP64 state without any
// device allocation.
//
// Some callers cannot call cudaMalloc: a host application whose device memory
// is owned by its own pool allocator (which forbids allocations behind its
// back), or one that fixes its device-memory budget at start-up and must not
// grow it later.  fvb_step_noalloc serves them: the caller passes its padded
// state; the two RK stage buffers and the step control this path needs live
// in one file-scope __device__ array of fixed size instead of memory from
// cudaMalloc.  That array is part of the library image, so every GPU that
// loads libfvb.so holds it (about 17 MB) until the process exits.
//
// The same stage kernel as fvb_step runs here, with plain (non-TMA) loads
// because the caller's IDX_P rows need not be 16-byte aligned.
#include "fvb_host.h"

namespace fvb {
namespace {

constexpr int kNoallocMaxN = 512;                 // largest grid side
constexpr int kNoallocMaxNp = kNoallocMaxN + 8;   // padded side for UP7 (g = 4)
constexpr size_t kPlanePad = (size_t)kNoallocMaxNp * kNoallocMaxNp;
constexpr size_t kCtrlDoubles = 32;               // 256 bytes for the step control
constexpr size_t kScratchDoubles = kCtrlDoubles + 2 * 4 * kPlanePad;

// step control, then the stage-1 and stage-2 outputs (4 planes each)
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Device address of the array in the CUDA context current on this thread.
// In host code the symbol is only a host-side stand-in, and the address
// belongs to one context: after cudaDeviceReset, or under a caller's own
// non-primary context on the same device, a cached address would be stale.
// So it is looked up on every call (a table lookup in the runtime, small
// next to the launches that follow).
fvb_status scratch_for_current_context(double **out)
{
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(scratch)");
    *out = (double *)p;
    return FVB_OK;
}

}  // namespace
}  // namespace fvb

using namespace fvb;

extern "C" fvb_status fvb_step_noalloc(double *Qp, int n, int np, double h, double cfl, double gamma, int bc_x,
                                       int bc_y, int nsteps, double t0, double t_stop, void *stream, fvb_stats *st)
{
    if (!Qp) return fail(FVB_ERR_INVALID, "null state");
    if (n < 4 || n > kNoallocMaxN)
        return fail(FVB_ERR_INVALID, "fvb_step_noalloc: n = %d outside [4, %d] (its fixed scratch holds grids "
                                     "up to %d x %d)", n, kNoallocMaxN, kNoallocMaxN, kNoallocMaxN);
    if (np < n + 8 || np > kNoallocMaxNp)
        return fail(FVB_ERR_INVALID, "fvb_step_noalloc: np = %d must be in [n + 8, %d]", np, kNoallocMaxNp);
    if (nsteps < 0 || bc_x < 0 || bc_x > 2 || bc_y < 0 || bc_y > 2 || !(h > 0) || !(cfl > 0) || !(gamma > 1))
        return fail(FVB_ERR_INVALID, "fvb_step_noalloc: bad step count, boundary condition, h, cfl or gamma");
    double *scratch = nullptr;
    fvb_status r = scratch_for_current_context(&scratch);
    if (r) return r;
    cudaStream_t s = (cudaStream_t)stream;

    StageArgs a{};
    GridDev &gd = a.grid;
    gd.n = n;
    gd.g = 4;
    gd.pitch = np;
    gd.xoff = 0;
    gd.plane = (long long)np * np;
    gd.bcx = bc_x;
    gd.bcy = bc_y;
    gd.h = h;
    gd.gam = gamma;
    gd.st[0] = Qp;
    gd.st[1] = nullptr;
    gd.lo[0] = gd.lo[1] = nullptr;
    gd.ctrl = (Ctrl *)scratch;
    gd.k1 = scratch + kCtrlDoubles;
    gd.k2 = scratch + kCtrlDoubles + 4 * (size_t)gd.plane;
    gd.tmap = nullptr;
    const int shape = 0;
    int tiles;
    tile_dims(shape, n, gd.tiles_x, tiles);
    int per_sm = stage_max_ctas_per_sm(P64, 7, shape), sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (per_sm <= 0 || sms <= 0) return fail(FVB_ERR_CUDA, "stage kernel cannot launch on this device");
    const int ctas = tiles < per_sm * sms ? tiles : per_sm * sms;

    // ghosts of the caller's state, max wave speed into the (cleared) step
    // control, then the step control itself: the array keeps whatever the
    // previous call left, so everything read before it is written is reset
    BufView v{n, 4, np, 0, gd.plane};
    cudaError_t e = bc_fill<double>(Qp, v, bc_x, bc_y, s);
    if (e == cudaSuccess) e = lam_into(Qp, v, INT_PRIM64, gamma, &gd.ctrl->lam_acc, s);
    if (e == cudaSuccess) e = ctrl_set(gd.ctrl, t_stop, 1, t0, cfl, h, s);
    a.ntiles_static = tiles;
    a.parity = 0;
    for (int k = 0; k < nsteps && e == cudaSuccess; ++k)
        for (int stage = 1; stage <= 3 && e == cudaSuccess; ++stage) {
            a.stage = stage;
            e = launch_stage(P64, 7, shape, a, ctas, s);
        }
    if (e != cudaSuccess) return cuda_fail(e, "fvb_step_noalloc");
    if (st) {
        Ctrl c;
        e = cudaMemcpyAsync(&c, gd.ctrl, sizeof c, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_fail(e, "fvb_step_noalloc: step control");
        *st = fvb_stats{};
        st->t = c.t;
        st->dt = c.dt;
        unsigned long long b = c.lam_acc;
        static_assert(sizeof b == sizeof st->lam_max, "lam bits");
        __builtin_memcpy(&st->lam_max, &b, sizeof b);
        st->t_stop = c.t_stop;
        st->steps = c.step;
        st->status = c.status;
    }
    return FVB_OK;
}
