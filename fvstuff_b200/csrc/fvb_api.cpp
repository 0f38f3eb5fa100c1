// fvb_api.cpp -- the single-grid solver behind the C ABI (include/fvb.h).
//
// A solver owns one device allocation holding its padded state buffers, the
// two stage buffers and its step control.  fvb_step enqueues three stage
// launches per step (or replays them as a CUDA graph) and never waits;
// dt, the CFL reduction and the stop test all live on the device, so the
// host synchronises only when it asks for the state or the step control.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "fvb_aux.h"
#include "fvb_host.h"

namespace fvb {

thread_local std::string g_err;

fvb_status fail(fvb_status st, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return st;
}

fvb_status cuda_fail(cudaError_t e, const char *what)
{
    return fail(FVB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

int prec_internal(int prec)
{
    return prec == FVB_PREC_F64 ? INT_PRIM64 : prec == FVB_PREC_F32 ? INT_PRIM32 : INT_CONS_HILO;
}

size_t prec_elem(int prec) { return prec == FVB_PREC_F64 ? 8 : 4; }

Geometry make_geometry(int n, int g, int prec)
{
    Geometry G{};
    const int align = 16;  // interior rows start 16 elements into a 16-aligned row
    G.n = n;
    G.g = g;
    G.np = n + 2 * g;
    G.xoff = align - g;
    G.pitch = ((G.xoff + G.np + align - 1) / align) * align;
    G.plane = (((long long)G.pitch * G.np + 63) / 64) * 64;
    G.elem = prec_elem(prec);
    G.nbuf = prec == FVB_PREC_F32C ? 6 : 3;
    G.bytes = (size_t)G.nbuf * 4 * G.plane * G.elem;
    return G;
}

void grid_pointers(GridDev &gd, void *base, const Geometry &G, int prec)
{
    char *p = (char *)base;
    size_t bb = (size_t)4 * G.plane * G.elem;
    gd.n = G.n;
    gd.g = G.g;
    gd.pitch = G.pitch;
    gd.xoff = G.xoff;
    gd.plane = G.plane;
    if (prec == FVB_PREC_F32C) {
        gd.st[0] = p; gd.st[1] = p + bb; gd.lo[0] = p + 2 * bb; gd.lo[1] = p + 3 * bb;
        gd.k1 = p + 4 * bb; gd.k2 = p + 5 * bb;
    } else {
        gd.st[0] = p; gd.st[1] = nullptr; gd.lo[0] = gd.lo[1] = nullptr;
        gd.k1 = p + bb; gd.k2 = p + 2 * bb;
    }
}

BufView view_of(const GridDev &gd) { return BufView{gd.n, gd.g, gd.pitch, gd.xoff, gd.plane}; }

void tile_dims(int shape, int n, int &tiles_x, int &tiles)
{
    const TileShape &t = kTileShapes[shape];
    tiles_x = (n + t.tx - 1) / t.tx;
    tiles = tiles_x * ((n + t.ty - 1) / t.ty);
}

void case_defaults(fvb_case *c, int kind, double x0, double y0, double L)
{
    std::memset(c, 0, sizeof *c);
    c->kind = kind;
    switch (kind) {
    case FVB_CASE_SOD:
        c->param[0] = x0 + 0.5 * L; c->param[1] = y0 + 0.5 * L; c->param[2] = 0.25 * L;
        c->param[3] = 0.125; c->param[4] = 11.0; c->param[5] = 0.1; c->param[6] = 10.0;
        break;
    case FVB_CASE_VORTEX:
        c->param[0] = 5.0; c->param[1] = 1.0; c->param[2] = 1.0;
        c->param[3] = x0 + 0.5 * L; c->param[4] = y0 + 0.5 * L;
        break;
    case FVB_CASE_KH:
        c->param[0] = y0 + 0.5 * L; c->param[1] = 0.25 * L; c->param[2] = 2.0; c->param[3] = 1.0;
        c->param[4] = -0.5; c->param[5] = 0.5; c->param[6] = 2.5; c->param[7] = 1e-3;
        c->seed = 12345;
        break;
    case FVB_CASE_RIEMANN4:
        c->param[0] = x0 + 0.5 * L; c->param[1] = y0 + 0.5 * L; c->param[2] = 2.0;
        c->seed = 1;
        break;
    case FVB_CASE_LMV:
        c->param[0] = 0.1;
        break;
    case FVB_CASE_UNIFORM:
        c->param[0] = 1.0; c->param[3] = 1.0;
        break;
    case FVB_CASE_GRESHO:
        c->param[0] = 0.1;  // eps (fv_rec3_2d.cu:511)
        break;
    default:
        break;
    }
}

}  // namespace fvb

using namespace fvb;

struct fvb_solver {
    fvb_config cfg;
    int prec = 0, order = 7, g = 4, n = 0;
    int internal = 0;
    Geometry G{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    void *block = nullptr;
    GridDev gd{};
    Ctrl *ctrl = nullptr;       // device
    Ctrl *ctrl_host = nullptr;  // pinned
    void *staging = nullptr;    // device, 4 (n+2g)^2 doubles
    double *sums_dev = nullptr, *sums_host = nullptr;
    int sums_blocks = 0;
    int shape = 0, tiles = 0, ctas = 0;
    int parity = 0;
    bool use_graph = false;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    int graph_steps = 1;
    bool keep = false;  // KEEP flux family: conserved FP64 state, g = 2
    bool rec3 = false;  // rec3 + Zhang-Shu family: conserved FP64 state, g = 2
    bool d2av = false;  // UP + HLLC + D2 viscosity (.bak): conserved FP64 state, g >= 3
    D2Params av{0.5, 0.0, 0.05};  // its C2, Cg, sc (fv_up7_ducros_2d.cu.bak:742-744)
    int rs = 0;         // solver on the reconstructed states: 0 HLLC, 1 HLL, 2 Roe
    // frame extraction (fvb_frame_begin / fvb_frame_end)
    float *frame_prim = nullptr;   // device, FP32 primitives with ghosts
    float *frame_dev = nullptr;    // device, 5 n x n fields
    float *frame_host = nullptr;   // pinned copy of them
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t frame_ready = nullptr, frame_copied = nullptr;
    bool frame_pending = false, frame_used = false;
    // posted step-control reads (fvb_stats_post / fvb_stats_wait)
    Ctrl *stats_ring = nullptr;  // pinned, FVB_STATS_SLOTS entries
    cudaEvent_t stats_ev[FVB_STATS_SLOTS] = {};
    bool stats_posted[FVB_STATS_SLOTS] = {};
};

static fvb_status ensure_staging(fvb_solver *s)
{
    if (s->staging) return FVB_OK;
    size_t bytes = (size_t)4 * s->G.np * s->G.np * sizeof(double);
    cudaError_t e = cudaMalloc(&s->staging, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(staging)");
    return FVB_OK;
}

static StageArgs stage_args(const fvb_solver *s, int stage, int parity)
{
    StageArgs a{};
    a.grid = s->gd;
    a.grids = nullptr;
    a.tiles = nullptr;
    a.ntiles = nullptr;
    a.ntiles_static = s->tiles;
    a.stage = stage;
    a.parity = parity;
    return a;
}

static cudaError_t enqueue_steps_direct(fvb_solver *s, int nsteps)
{
    for (int k = 0; k < nsteps; ++k) {
        if (s->keep || s->rec3 || s->d2av) {
            for (int stage = 1; stage <= 3; ++stage) {
                cudaError_t e = s->keep   ? keep_launch_stage(s->gd, stage, s->tiles, s->stream)
                                : s->rec3 ? rec3_launch_stage(s->gd, stage, s->tiles, s->stream)
                                          : d2av_launch_stage(s->gd, s->order, stage, s->tiles, s->av, s->stream);
                if (e != cudaSuccess) return e;
            }
            continue;
        }
        for (int stage = 1; stage <= 3; ++stage) {
            StageArgs a = stage_args(s, stage, s->parity);
            cudaError_t e = launch_stage(s->prec, s->order, s->shape, a, s->ctas, s->stream, s->rs);
            if (e != cudaSuccess) return e;
        }
        if (s->prec == FVB_PREC_F32C) s->parity ^= 1;
    }
    return cudaSuccess;
}

static void drop_graphs(fvb_solver *s)
{
    for (auto &g : s->gexec)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

static cudaError_t capture_graph(fvb_solver *s, int parity)
{
    cudaGraph_t graph = nullptr;
    int saved = s->parity;
    s->parity = parity;
    cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { s->parity = saved; return e; }
    cudaError_t el = enqueue_steps_direct(s, s->graph_steps);
    e = cudaStreamEndCapture(s->stream, &graph);
    s->parity = saved;
    if (el != cudaSuccess) { if (graph) cudaGraphDestroy(graph); return el; }
    if (e != cudaSuccess) return e;
    e = cudaGraphInstantiate(&s->gexec[parity], graph, 0);
    cudaGraphDestroy(graph);
    return e;
}

static cudaError_t enqueue_steps(fvb_solver *s, int nsteps)
{
    if (!s->use_graph) return enqueue_steps_direct(s, nsteps);
    while (nsteps >= s->graph_steps) {
        int p = s->parity;
        if (!s->gexec[p]) {
            cudaError_t e = capture_graph(s, p);
            if (e != cudaSuccess) return e;
        }
        cudaError_t e = cudaGraphLaunch(s->gexec[p], s->stream);
        if (e != cudaSuccess) return e;
        nsteps -= s->graph_steps;
        // a graph of an even number of F32C steps ends on its start parity
    }
    return enqueue_steps_direct(s, nsteps);
}

static fvb_status refresh_after_state(fvb_solver *s, int buf_parity)
{
    cudaError_t e;
    BufView v = view_of(s->gd);
    if (s->rec3) {
        // as fv_rec3 after its initial state: the limiter pass, then ghosts
        e = cudaMemsetAsync(&s->ctrl->aux, 0, sizeof(unsigned long long), s->stream);
        if (e == cudaSuccess) e = rec3_limit_into(s->gd, s->gd.st[0], s->stream);
        if (e == cudaSuccess) e = bc_fill<double>((double *)s->gd.st[0], v, s->gd.bcx, s->gd.bcy, s->stream);
        if (e == cudaSuccess) e = rec3_lam_into(s->gd, s->stream);
        if (e == cudaSuccess) e = ctrl_set(s->ctrl, 0.0, 1, 0.0, s->cfg.cfl, s->cfg.length / s->n, s->stream);
        return e == cudaSuccess ? FVB_OK : cuda_fail(e, "state refresh");
    }
    if (s->keep || s->d2av) {
        e = bc_fill<double>((double *)s->gd.st[0], v, s->gd.bcx, s->gd.bcy, s->stream);
        if (e == cudaSuccess) e = s->keep ? keep_lam_into(s->gd, s->stream) : d2av_lam_into(s->gd, s->stream);
        if (e == cudaSuccess) e = ctrl_set(s->ctrl, 0.0, 1, 0.0, s->cfg.cfl, s->cfg.length / s->n, s->stream);
        return e == cudaSuccess ? FVB_OK : cuda_fail(e, "state refresh");
    }
    if (s->internal == INT_PRIM64) e = bc_fill<double>((double *)s->gd.st[0], v, s->gd.bcx, s->gd.bcy, s->stream);
    else if (s->internal == INT_PRIM32) e = bc_fill<float>((float *)s->gd.st[0], v, s->gd.bcx, s->gd.bcy, s->stream);
    else {
        e = bc_fill<float>((float *)s->gd.st[buf_parity], v, s->gd.bcx, s->gd.bcy, s->stream);
        if (e == cudaSuccess) e = bc_fill<float>((float *)s->gd.lo[buf_parity], v, s->gd.bcx, s->gd.bcy, s->stream);
    }
    if (e != cudaSuccess) return cuda_fail(e, "ghost fill");
    e = lam_into(s->gd.st[s->internal == INT_CONS_HILO ? buf_parity : 0], v, s->internal, s->cfg.gamma,
                 &s->ctrl->lam_acc, s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "max wave speed");
    e = ctrl_set(s->ctrl, 0.0, 1, 0.0, s->cfg.cfl, s->cfg.length / s->n, s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "step control reset");
    return FVB_OK;
}

extern "C" {

const char *fvb_version(void) { return "fvb 0.1 (sm_100a)"; }

const char *fvb_device_name(int device)
{
    thread_local std::string name;
    cudaDeviceProp prop;
    const cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) {
        cuda_fail(e, "cudaGetDeviceProperties");
        return nullptr;
    }
    name = prop.name;
    return name.c_str();
}

const char *fvb_last_error(void) { return g_err.c_str(); }

void fvb_config_default(fvb_config *c, int n)
{
    std::memset(c, 0, sizeof *c);
    c->n = n;
    c->order = 7;
    c->flux = FVB_FLUX_UP_DUCROS;
    c->precision = FVB_PREC_F64;
    c->bc_x = c->bc_y = FVB_BC_REFLECT;
    c->x0 = 0.0;
    c->y0 = 0.0;
    c->length = 1.0;
    c->gamma = 1.4;
    c->cfl = 0.4;
    c->device = 0;
    c->stream = nullptr;
    c->tile = -1;
}

void fvb_case_default(fvb_case *c, int kind, double x0, double y0, double length)
{
    case_defaults(c, kind, x0, y0, length);
}

fvb_status fvb_create(const fvb_config *cfg, fvb_solver **out)
{
    if (!cfg || !out) return fail(FVB_ERR_INVALID, "null argument");
    *out = nullptr;
    const bool keep = cfg->flux == FVB_FLUX_KEEP;
    const bool rec3 = cfg->flux == FVB_FLUX_REC3;
    const bool d2av = cfg->flux == FVB_FLUX_UP_HLLC_D2AV;
    const int rs = cfg->flux == FVB_FLUX_UP_DUCROS_HLL ? 1 : cfg->flux == FVB_FLUX_UP_DUCROS_ROE ? 2 : 0;
    if (cfg->flux != FVB_FLUX_UP_DUCROS && !keep && !rec3 && !d2av && rs == 0)
        return fail(FVB_ERR_INVALID, "unknown flux %d", cfg->flux);
    if (d2av && cfg->precision != FVB_PREC_F64)
        return fail(FVB_ERR_INVALID, "the UP + HLLC + D2 viscosity scheme runs in FP64 (as fv_up7_ducros_2d.cu.bak)");
    if (rec3 && (cfg->precision != FVB_PREC_F64 || cfg->bc_x != FVB_BC_PERIODIC || cfg->bc_y != FVB_BC_PERIODIC ||
                 cfg->n % 2))
        return fail(FVB_ERR_INVALID, "the rec3 family runs in FP64 on periodic grids of even n (as fv_rec3_2d.cu)");
    if (rs && !(cfg->precision == FVB_PREC_F64 && cfg->order == 7))
        return fail(FVB_ERR_INVALID, "the HLL / Roe variants are built for FP64, order 7");
    if (cfg->precision < 0 || cfg->precision > 2) return fail(FVB_ERR_INVALID, "unknown precision %d", cfg->precision);
    if (keep && cfg->precision != FVB_PREC_F64)
        return fail(FVB_ERR_INVALID, "the KEEP flux family runs in FP64 (as keep_fv_euler_2d.cu)");
    if (!keep && !rec3 && !(cfg->order == 3 || cfg->order == 5 || cfg->order == 7 || cfg->order == 9))
        return fail(FVB_ERR_INVALID, "order must be 3, 5, 7 or 9 (got %d)", cfg->order);
    if (!keep && !rec3 && cfg->precision != FVB_PREC_F64 && cfg->order != 7)
        return fail(FVB_ERR_INVALID, "orders 3, 5 and 9 are built for FP64 only");
    const int g = (keep || rec3) ? 2 : d2av ? d2av_ghost(cfg->order) : (cfg->order + 1) / 2;
    if (cfg->n < g || cfg->n > 65536) return fail(FVB_ERR_INVALID, "n = %d out of range [%d, 65536]", cfg->n, g);
    for (int b : {cfg->bc_x, cfg->bc_y})
        if (b < 0 || b > 2) return fail(FVB_ERR_INVALID, "unknown boundary condition %d", b);
    if (!(cfg->length > 0) || !(cfg->cfl > 0) || !(cfg->gamma > 1))
        return fail(FVB_ERR_INVALID, "length, cfl must be > 0 and gamma > 1");
    if (cfg->tile >= kNumTileShapes) return fail(FVB_ERR_INVALID, "tile variant %d out of range", cfg->tile);

    cudaError_t e = cudaSetDevice(cfg->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");

    fvb_solver *s = new fvb_solver();
    s->cfg = *cfg;
    s->prec = cfg->precision;
    s->order = cfg->order;
    s->g = g;
    s->n = cfg->n;
    s->keep = keep;
    s->rec3 = rec3;
    s->d2av = d2av;
    s->rs = rs;
    s->internal = (keep || rec3 || d2av) ? INT_CONS64 : prec_internal(s->prec);
    s->G = make_geometry(cfg->n, g, s->prec);
    if (cfg->stream) s->stream = (cudaStream_t)cfg->stream;
    else {
        e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) { delete s; return cuda_fail(e, "cudaStreamCreate"); }
        s->own_stream = true;
    }
    // buffers | step control | TMA descriptors (64-byte aligned)
    const size_t ctrl_off = (s->G.bytes + 255) / 256 * 256;
    const size_t tmap_off = ctrl_off + 256;
    size_t total = tmap_off + TM_COUNT * sizeof(CUtensorMap);
    e = cudaMalloc(&s->block, total);
    if (e != cudaSuccess) {
        fvb_destroy(s);
        return fail(FVB_ERR_NOMEM, "cudaMalloc(%zu bytes): %s", total, cudaGetErrorString(e));
    }
    e = cudaMemsetAsync(s->block, 0, total, s->stream);
    if (e != cudaSuccess) { fvb_destroy(s); return cuda_fail(e, "cudaMemset"); }
    grid_pointers(s->gd, s->block, s->G, s->prec);
    s->ctrl = (Ctrl *)((char *)s->block + ctrl_off);
    s->gd.ctrl = s->ctrl;
    s->gd.tmap = nullptr;
    s->gd.bcx = cfg->bc_x;
    s->gd.bcy = cfg->bc_y;
    s->gd.h = cfg->length / cfg->n;
    s->gd.gam = cfg->gamma;
    e = cudaMallocHost(&s->ctrl_host, sizeof(Ctrl));
    if (e != cudaSuccess) { fvb_destroy(s); return cuda_fail(e, "cudaMallocHost"); }

    if (keep || rec3 || d2av) {
        // KEEP / rec3 / D2 viscosity: plain loads into their own tile kernels
        if (keep) keep_tiles(s->n, s->gd.tiles_x, s->tiles);
        else if (rec3) rec3_tiles(s->n, s->gd.tiles_x, s->tiles);
        else d2av_tiles(s->n, s->gd.tiles_x, s->tiles);
        s->graph_steps = 1;
        s->use_graph = cfg->n <= 512;
        e = ctrl_set(s->ctrl, 0.0, 1, 0.0, cfg->cfl, s->gd.h, s->stream);
        if (e != cudaSuccess) { fvb_destroy(s); return cuda_fail(e, "step control"); }
        *out = s;
        return FVB_OK;
    }
    s->shape = cfg->tile >= 0 ? cfg->tile : autotune_shape(s->prec, s->order, cfg->n);
    tile_dims(s->shape, s->n, s->gd.tiles_x, s->tiles);
    {
        CUtensorMap maps[TM_COUNT];
        if (encode_tile_maps(s->gd, s->prec, s->order, s->shape, maps)) {
            CUtensorMap *dmaps = (CUtensorMap *)((char *)s->block + tmap_off);
            e = cudaMemcpyAsync(dmaps, maps, sizeof maps, cudaMemcpyHostToDevice, s->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
            if (e != cudaSuccess) { fvb_destroy(s); return cuda_fail(e, "tensor maps"); }
            s->gd.tmap = dmaps;
        }
    }
    {
        int per_sm = stage_max_ctas_per_sm(s->prec, s->order, s->shape, s->rs), sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cfg->device);
        s->ctas = std::min(s->tiles, std::max(1, per_sm) * std::max(1, sms));
    }
    s->graph_steps = s->prec == FVB_PREC_F32C ? 2 : 1;
    s->use_graph = cfg->n <= 512;
    e = ctrl_set(s->ctrl, 0.0, 1, 0.0, cfg->cfl, s->gd.h, s->stream);
    if (e != cudaSuccess) { fvb_destroy(s); return cuda_fail(e, "step control"); }
    // make sure the kernel variant can launch on this device
    if (stage_max_ctas_per_sm(s->prec, s->order, s->shape, s->rs) <= 0) {
        fvb_destroy(s);
        return fail(FVB_ERR_CUDA, "stage kernel variant cannot be resident on this device");
    }
    *out = s;
    return FVB_OK;
}

void fvb_destroy(fvb_solver *s)
{
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    drop_graphs(s);
    if (s->block) cudaFree(s->block);
    if (s->staging) cudaFree(s->staging);
    if (s->sums_dev) cudaFree(s->sums_dev);
    if (s->sums_host) cudaFreeHost(s->sums_host);
    if (s->ctrl_host) cudaFreeHost(s->ctrl_host);
    if (s->copy_stream) cudaStreamSynchronize(s->copy_stream);
    if (s->frame_prim) cudaFree(s->frame_prim);
    if (s->frame_dev) cudaFree(s->frame_dev);
    if (s->frame_host) cudaFreeHost(s->frame_host);
    if (s->frame_ready) cudaEventDestroy(s->frame_ready);
    if (s->frame_copied) cudaEventDestroy(s->frame_copied);
    if (s->stats_ring) cudaFreeHost(s->stats_ring);
    for (cudaEvent_t ev : s->stats_ev)
        if (ev) cudaEventDestroy(ev);
    if (s->copy_stream) cudaStreamDestroy(s->copy_stream);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

int fvb_ghost_width(const fvb_solver *s) { return s ? s->g : 0; }

fvb_status fvb_init_case(fvb_solver *s, const fvb_case *c)
{
    NvtxRange nvtx_range("fvb_init_case");
    if (!s || !c) return fail(FVB_ERR_INVALID, "null argument");
    if (c->kind >= FVB_CASE_REC3_SOD && c->kind <= FVB_CASE_GRESHO) {
        if (!s->rec3) return fail(FVB_ERR_INVALID, "case %d is a rec3 case (FVB_FLUX_REC3)", c->kind);
        const double eps = c->param[0] > 0 ? c->param[0] : 0.1;
        const double p0 = 1.0 / (s->cfg.gamma * eps * eps) - 0.5;  // fv_rec3_2d.cu:518
        cudaError_t e = rec3_init_case(s->gd, c->kind - FVB_CASE_REC3_SOD, p0, s->stream);
        if (e != cudaSuccess) return cuda_fail(e, "initial state");
        return refresh_after_state(s, 0);
    }
    fvb_status st = ensure_staging(s);
    if (st) return st;
    // the FP32 form as shipped starts its Sod from the FP32 evaluation
    const bool sod32 = s->prec == P32 && c->kind == FVB_CASE_SOD;
    cudaError_t e = sod32 ? init_sod_prim32((float *)s->staging, s->n, s->cfg.x0, s->cfg.y0, s->cfg.length, *c,
                                            s->stream)
                          : init_case_prim64((double *)s->staging, s->n, s->cfg.x0, s->cfg.y0, s->gd.h,
                                             s->cfg.gamma, *c, s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "initial state");
    ExtView ev{1, s->g, s->G.np, FVB_LAYOUT_PRIM, sod32 ? FVB_F32 : FVB_F64};
    int p = s->parity;
    e = import_state(s->staging, ev, s->gd.st[s->internal == INT_CONS_HILO ? p : 0], s->gd.lo[p], view_of(s->gd),
                     s->internal, s->cfg.gamma, s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "import");
    return refresh_after_state(s, p);
}

fvb_status fvb_set_state(fvb_solver *s, const void *src, int layout, int dtype, int where, int interior_only)
{
    NvtxRange nvtx_range("fvb_set_state");
    if (!s || !src) return fail(FVB_ERR_INVALID, "null argument");
    if ((layout != 0 && layout != 1) || (dtype != 0 && dtype != 1) || (where != 0 && where != 1))
        return fail(FVB_ERR_INVALID, "bad layout/dtype/where");
    ExtView ev{interior_only ? 1 : 0, s->g, s->G.np, layout, dtype};
    const void *dev = src;
    if (where == FVB_HOST) {
        fvb_status st = ensure_staging(s);
        if (st) return st;
        long long side = interior_only ? s->n : s->G.np;
        size_t bytes = (size_t)4 * side * side * (dtype == FVB_F64 ? 8 : 4);
        cudaError_t e = cudaMemcpyAsync(s->staging, src, bytes, cudaMemcpyHostToDevice, s->stream);
        if (e != cudaSuccess) return cuda_fail(e, "copy in");
        dev = s->staging;
    }
    int p = s->parity;
    cudaError_t e = import_state(dev, ev, s->gd.st[s->internal == INT_CONS_HILO ? p : 0], s->gd.lo[p],
                                 view_of(s->gd), s->internal, s->cfg.gamma, s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "import");
    fvb_status st = refresh_after_state(s, p);
    if (st) return st;
    if (where == FVB_HOST) {
        e = cudaStreamSynchronize(s->stream);  // the caller may reuse its buffer on return
        if (e != cudaSuccess) return cuda_fail(e, "sync");
    }
    return FVB_OK;
}

fvb_status fvb_get_state(fvb_solver *s, void *dst, int layout, int dtype, int where, int interior_only)
{
    NvtxRange nvtx_range("fvb_get_state");
    if (!s || !dst) return fail(FVB_ERR_INVALID, "null argument");
    if ((layout != 0 && layout != 1) || (dtype != 0 && dtype != 1) || (where != 0 && where != 1))
        return fail(FVB_ERR_INVALID, "bad layout/dtype/where");
    ExtView ev{interior_only ? 1 : 0, s->g, s->G.np, layout, dtype};
    void *dev = dst;
    if (where == FVB_HOST) {
        fvb_status st = ensure_staging(s);
        if (st) return st;
        dev = s->staging;
    }
    int p = s->parity;
    cudaError_t e = export_state(s->gd.st[s->internal == INT_CONS_HILO ? p : 0], s->gd.lo[p], view_of(s->gd),
                                 s->internal, dev, ev, s->cfg.gamma, s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "export");
    if (where == FVB_HOST) {
        long long side = interior_only ? s->n : s->G.np;
        size_t bytes = (size_t)4 * side * side * (dtype == FVB_F64 ? 8 : 4);
        e = cudaMemcpyAsync(dst, s->staging, bytes, cudaMemcpyDeviceToHost, s->stream);
        if (e != cudaSuccess) return cuda_fail(e, "copy out");
        e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) return cuda_fail(e, "sync");
    }
    return FVB_OK;
}

fvb_status fvb_limiter_fixes(fvb_solver *s, int64_t *count)
{
    if (!s || !count) return fail(FVB_ERR_INVALID, "null argument");
    *count = 0;
    if (!s->rec3) return FVB_OK;  // aux holds other families' own quantities
    unsigned long long v = 0;
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e == cudaSuccess) e = cudaMemcpy(&v, &s->ctrl->aux, sizeof v, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "limiter count");
    *count = (int64_t)v;
    return FVB_OK;
}

fvb_status fvb_set_d2av(fvb_solver *s, double c2, double cg, double sc)
{
    if (!s) return fail(FVB_ERR_INVALID, "null argument");
    if (!s->d2av) return fail(FVB_ERR_INVALID, "the solver does not use FVB_FLUX_UP_HLLC_D2AV");
    if (!(c2 >= 0) || !(cg >= 0) || !(sc >= 0)) return fail(FVB_ERR_INVALID, "C2, Cg and sc must be >= 0");
    s->av = D2Params{c2, cg, sc};
    drop_graphs(s);  // the kernels take the coefficients as arguments
    return FVB_OK;
}

fvb_status fvb_debug_drop_load(fvb_solver *s)
{
    if (!s) return fail(FVB_ERR_INVALID, "null argument");
    if (s->keep || s->rec3 || s->d2av || !s->gd.tmap)
        return fail(FVB_ERR_INVALID, "the hook needs a TMA-fed UP grid");
    static const int one = 1;
    cudaError_t e = cudaMemcpyAsync(&s->ctrl->drop_load, &one, sizeof one, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    return e == cudaSuccess ? FVB_OK : cuda_fail(e, "arm");
}

// ---- frames: extraction on the device, copy on a second stream ----------

fvb_status fvb_frame_begin(fvb_solver *s)
{
    NvtxRange nvtx_range("fvb_frame_begin");
    if (!s) return fail(FVB_ERR_INVALID, "null argument");
    const size_t n2 = (size_t)s->n * s->n, np2 = (size_t)s->G.np * s->G.np;
    cudaError_t e = cudaSuccess;
    if (!s->frame_dev) {
        e = cudaMalloc(&s->frame_prim, 4 * np2 * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&s->frame_dev, 5 * n2 * sizeof(float));
        if (e == cudaSuccess) e = cudaMallocHost(&s->frame_host, 5 * n2 * sizeof(float));
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->frame_ready, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->frame_copied, cudaEventDisableTiming);
        if (e != cudaSuccess) return cuda_fail(e, "frame buffers");
    }
    // the previous frame's copy must be done before its buffers are reused
    if (s->frame_used) e = cudaStreamWaitEvent(s->stream, s->frame_copied, 0);
    ExtView ev{0, s->g, s->G.np, FVB_LAYOUT_PRIM, FVB_F32};
    const int p = s->parity;
    if (e == cudaSuccess)
        e = export_state(s->gd.st[s->internal == INT_CONS_HILO ? p : 0], s->gd.lo[p], view_of(s->gd), s->internal,
                         s->frame_prim, ev, s->cfg.gamma, s->stream);
    if (e == cudaSuccess) e = frame_fields(s->frame_prim, s->n, s->g, s->G.np, s->gd.h, s->frame_dev, s->stream);
    // the .bak scheme's sensor panel is its own velocity-divergence weight
    if (e == cudaSuccess && s->d2av) e = d2av_sensor_into(s->gd, s->av.sc, s->frame_dev + 2 * n2, s->stream);
    if (e == cudaSuccess) e = cudaEventRecord(s->frame_ready, s->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s->copy_stream, s->frame_ready, 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->frame_host, s->frame_dev, 5 * n2 * sizeof(float), cudaMemcpyDeviceToHost,
                            s->copy_stream);
    if (e == cudaSuccess) e = cudaEventRecord(s->frame_copied, s->copy_stream);
    if (e != cudaSuccess) return cuda_fail(e, "frame");
    s->frame_pending = s->frame_used = true;
    return FVB_OK;
}

fvb_status fvb_frame_end(fvb_solver *s, float *out)
{
    if (!s || !out) return fail(FVB_ERR_INVALID, "null argument");
    if (!s->frame_pending) return fail(FVB_ERR_INVALID, "no frame begun");
    cudaError_t e = cudaEventSynchronize(s->frame_copied);
    if (e != cudaSuccess) return cuda_fail(e, "frame copy");
    std::memcpy(out, s->frame_host, (size_t)5 * s->n * s->n * sizeof(float));
    s->frame_pending = false;
    return FVB_OK;
}

// checkpoint file: a fixed header, then the current state buffer(s) as
// stored on the device (pitched padded planes), so a load is exact
struct CkptHeader {
    char magic[8];  // "FVBCKPT1"
    int n, g, order, flux, precision, internal;
    long long plane;
    int pitch, xoff;
    double t;
    long long steps;
    unsigned long long lam_bits;
    int nbufs, pad;
};

fvb_status fvb_save(fvb_solver *s, const char *path)
{
    if (!s || !path) return fail(FVB_ERR_INVALID, "null argument");
    fvb_stats st;
    fvb_status r = fvb_sync(s, &st);
    if (r) return r;
    CkptHeader h{};
    std::memcpy(h.magic, "FVBCKPT1", 8);
    h.n = s->n; h.g = s->g; h.order = s->order; h.flux = s->cfg.flux; h.precision = s->prec;
    h.internal = s->internal; h.plane = s->G.plane; h.pitch = s->G.pitch; h.xoff = s->G.xoff;
    h.t = s->ctrl_host->t; h.steps = s->ctrl_host->step; h.lam_bits = s->ctrl_host->lam_acc;
    h.nbufs = s->internal == INT_CONS_HILO ? 2 : 1;
    const size_t bytes = (size_t)4 * s->G.plane * s->G.elem;
    std::vector<char> buf(bytes);
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(FVB_ERR_INVALID, "cannot open %s for writing", path);
    bool ok = std::fwrite(&h, sizeof h, 1, f) == 1;
    void *src[2] = {s->gd.st[s->internal == INT_CONS_HILO ? s->parity : 0], s->gd.lo[s->parity]};
    for (int b = 0; ok && b < h.nbufs; ++b) {
        cudaError_t e = cudaMemcpy(buf.data(), src[b], bytes, cudaMemcpyDeviceToHost);
        ok = e == cudaSuccess && std::fwrite(buf.data(), 1, bytes, f) == bytes;
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? FVB_OK : fail(FVB_ERR_INVALID, "writing %s failed", path);
}

fvb_status fvb_load(fvb_solver *s, const char *path)
{
    if (!s || !path) return fail(FVB_ERR_INVALID, "null argument");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(FVB_ERR_INVALID, "cannot open %s", path);
    CkptHeader h{};
    if (std::fread(&h, sizeof h, 1, f) != 1 || std::memcmp(h.magic, "FVBCKPT1", 8) != 0) {
        std::fclose(f);
        return fail(FVB_ERR_INVALID, "%s is not an fvb checkpoint", path);
    }
    if (h.n != s->n || h.g != s->g || h.order != s->order || h.flux != s->cfg.flux || h.precision != s->prec ||
        h.internal != s->internal || h.plane != s->G.plane || h.pitch != s->G.pitch) {
        std::fclose(f);
        return fail(FVB_ERR_INVALID, "checkpoint %s was written by a solver of another configuration", path);
    }
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) { std::fclose(f); return cuda_fail(e, "sync"); }
    const size_t bytes = (size_t)4 * s->G.plane * s->G.elem;
    std::vector<char> buf(bytes);
    void *dst[2] = {s->gd.st[s->internal == INT_CONS_HILO ? s->parity : 0], s->gd.lo[s->parity]};
    for (int b = 0; b < h.nbufs; ++b) {
        if (std::fread(buf.data(), 1, bytes, f) != bytes) { std::fclose(f); return fail(FVB_ERR_INVALID, "%s is truncated", path); }
        e = cudaMemcpy(dst[b], buf.data(), bytes, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { std::fclose(f); return cuda_fail(e, "restore"); }
    }
    std::fclose(f);
    // the step control as it was: time, steps, and the wave-speed max
    e = ctrl_set(s->ctrl, 0.0, 1, h.t, s->cfg.cfl, s->gd.h, s->stream);
    Ctrl c{};
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->ctrl_host, s->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "restore step control");
    c = *s->ctrl_host;
    c.step = h.steps;
    c.lam_acc = h.lam_bits;
    c.t = h.t;
    e = cudaMemcpy(s->ctrl, &c, sizeof c, cudaMemcpyHostToDevice);
    return e == cudaSuccess ? FVB_OK : cuda_fail(e, "restore step control");
}

fvb_status fvb_get_state_hilo(fvb_solver *s, float *hi, float *lo)
{
    if (!s || !hi || !lo) return fail(FVB_ERR_INVALID, "null argument");
    if (s->internal != INT_CONS_HILO) return fail(FVB_ERR_INVALID, "solver is not in the compensated FP32 mode");
    size_t row = (size_t)s->n * sizeof(float);
    int p = s->parity;
    for (int q = 0; q < 4; ++q) {
        size_t off = ((size_t)q * s->G.plane + (size_t)s->g * s->G.pitch + s->g + s->G.xoff) * sizeof(float);
        cudaError_t e = cudaMemcpy2DAsync(hi + (size_t)q * s->n * s->n, row, (char *)s->gd.st[p] + off,
                                          s->G.pitch * sizeof(float), row, s->n, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(lo + (size_t)q * s->n * s->n, row, (char *)s->gd.lo[p] + off,
                                  s->G.pitch * sizeof(float), row, s->n, cudaMemcpyDeviceToHost, s->stream);
        if (e != cudaSuccess) return cuda_fail(e, "copy out");
    }
    cudaError_t e = cudaStreamSynchronize(s->stream);
    return e == cudaSuccess ? FVB_OK : cuda_fail(e, "sync");
}

fvb_status fvb_step(fvb_solver *s, int nsteps, double t_stop)
{
    NvtxRange nvtx_range("fvb_step");
    if (!s || nsteps < 0) return fail(FVB_ERR_INVALID, "bad argument");
    cudaError_t e = ctrl_set(s->ctrl, t_stop, 0, 0, 0, 0, s->stream);
    if (e == cudaSuccess) e = enqueue_steps(s, nsteps);
    if (e != cudaSuccess) return cuda_fail(e, "step launch");
    return FVB_OK;
}

static void stats_from_ctrl(const Ctrl &c, fvb_stats *st)
{
    std::memset(st, 0, sizeof *st);
    st->t = c.t;
    st->dt = c.dt;
    unsigned long long b = c.lam_acc;
    std::memcpy(&st->lam_max, &b, sizeof b);
    st->t_stop = c.t_stop;
    st->steps = c.step;
    st->status = c.status;
}

fvb_status fvb_sync(fvb_solver *s, fvb_stats *st)
{
    if (!s) return fail(FVB_ERR_INVALID, "null solver");
    cudaError_t e = cudaMemcpyAsync(s->ctrl_host, s->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "sync");
    if (st) stats_from_ctrl(*s->ctrl_host, st);
    return FVB_OK;
}

fvb_status fvb_stats_post(fvb_solver *s, int slot)
{
    if (!s || slot < 0 || slot >= FVB_STATS_SLOTS) return fail(FVB_ERR_INVALID, "null solver or bad slot %d", slot);
    cudaError_t e = cudaSuccess;
    if (!s->stats_ring) e = cudaMallocHost(&s->stats_ring, sizeof(Ctrl) * FVB_STATS_SLOTS);
    if (e == cudaSuccess && !s->stats_ev[slot]) e = cudaEventCreateWithFlags(&s->stats_ev[slot], cudaEventDisableTiming);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->stats_ring + slot, s->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s->stream);
    if (e == cudaSuccess) e = cudaEventRecord(s->stats_ev[slot], s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "stats post");
    s->stats_posted[slot] = true;
    return FVB_OK;
}

fvb_status fvb_stats_wait(fvb_solver *s, int slot, fvb_stats *st)
{
    if (!s || !st || slot < 0 || slot >= FVB_STATS_SLOTS) return fail(FVB_ERR_INVALID, "bad argument");
    if (!s->stats_posted[slot]) return fail(FVB_ERR_INVALID, "nothing posted to slot %d", slot);
    const cudaError_t e = cudaEventSynchronize(s->stats_ev[slot]);
    if (e != cudaSuccess) return cuda_fail(e, "stats wait");
    stats_from_ctrl(s->stats_ring[slot], st);
    return FVB_OK;
}

fvb_status fvb_advance(fvb_solver *s, double t_stop, int64_t max_steps, int chunk)
{
    NvtxRange nvtx_range("fvb_advance");
    if (!s) return fail(FVB_ERR_INVALID, "null solver");
    int64_t done = 0;
    for (;;) {
        fvb_stats st;
        fvb_status r = fvb_sync(s, &st);
        if (r) return r;
        if (st.status) return fail((fvb_status)st.status, "step control stopped at t=%.9g step %lld (%s)", st.t,
                                   (long long)st.steps, st.status == FVB_ERR_BLOWUP ? "lam_max not > 0" : "dt underflow");
        // (the FP32 form's time is a float: it stops at the float t_stop)
        const bool before = s->prec == P32 ? (float)st.t < (float)t_stop : st.t < t_stop;
        if (!before || done >= max_steps) return FVB_OK;
        int64_t k = chunk;
        if (k <= 0) {
            double dt = st.lam_max > 0 ? s->cfg.cfl * (s->cfg.length / s->n) / st.lam_max : 0;
            double est = dt > 0 ? (t_stop - st.t) / dt : 1e9;
            k = (int64_t)std::min(est * 1.05 + 2.0, 4096.0);
            if (k < 1) k = 1;
        }
        if (k > max_steps - done) k = max_steps - done;
        r = fvb_step(s, (int)k, t_stop);
        if (r) return r;
        done += k;
    }
}

fvb_status fvb_stats_sums(fvb_solver *s, fvb_stats *st)
{
    if (!s || !st) return fail(FVB_ERR_INVALID, "null argument");
    if (!s->sums_dev) {
        s->sums_blocks = 592;
        cudaError_t e = cudaMalloc(&s->sums_dev, sizeof(double) * 5 * s->sums_blocks);
        if (e == cudaSuccess) e = cudaMallocHost(&s->sums_host, sizeof(double) * 5 * s->sums_blocks);
        if (e != cudaSuccess) return cuda_fail(e, "sums buffers");
    }
    int p = s->parity;
    cudaError_t e = sums_partials(s->gd.st[s->internal == INT_CONS_HILO ? p : 0], s->gd.lo[p], view_of(s->gd),
                                  s->internal, s->cfg.gamma, s->sums_dev, s->sums_blocks, s->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->sums_host, s->sums_dev, sizeof(double) * 5 * s->sums_blocks, cudaMemcpyDeviceToHost,
                            s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "sums");
    fvb_status r = fvb_sync(s, st);
    if (r) return r;
    double acc[5] = {0, 0, 0, 0, 0};
    for (int b = 0; b < s->sums_blocks; ++b)
        for (int q = 0; q < 5; ++q) acc[q] += s->sums_host[b * 5 + q];
    double h2 = s->gd.h * s->gd.h;
    for (int q = 0; q < 4; ++q) st->sums[q] = acc[q] * h2;
    st->nonfinite = acc[4] > 0;
    return FVB_OK;
}

fvb_status fvb_set_graph(fvb_solver *s, int enable)
{
    if (!s) return fail(FVB_ERR_INVALID, "null solver");
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return cuda_fail(e, "sync");
    s->use_graph = enable != 0;
    if (!s->use_graph) drop_graphs(s);
    return FVB_OK;
}

// ---- kernel-level contract ---------------------------------------------

fvb_status fvb_up_rhs(const void *Qp, void *rhs, void *lam, int n, int np, int order, double h, double gamma,
                      int dtype, void *stream)
{
    if (!Qp || !rhs || !lam) return fail(FVB_ERR_INVALID, "null argument");
    if (order != 7 && !(dtype == FVB_F64 && (order == 3 || order == 5 || order == 9)))
        return fail(FVB_ERR_INVALID, "order %d not built for this dtype", order);
    const int g = (order + 1) / 2;
    if (n < 1 || np < n + 2 * g) return fail(FVB_ERR_INVALID, "np must be >= n + 2g");
    StageArgs a{};
    GridDev &gd = a.grid;
    gd.n = n;
    gd.g = g;
    gd.pitch = np;
    gd.xoff = 0;
    gd.plane = (long long)np * np;
    gd.h = h;
    gd.gam = gamma;
    gd.st[0] = (void *)Qp;
    gd.ctrl = nullptr;
    const int shape = 0;
    int tiles;
    tile_dims(shape, n, gd.tiles_x, tiles);
    a.ntiles_static = tiles;
    a.stage = 0;
    a.rhs = rhs;
    a.lam = lam;
    int prec = dtype == FVB_F64 ? P64 : P32;
    cudaError_t e = launch_stage(prec, order, shape, a, tiles, (cudaStream_t)stream);
    return e == cudaSuccess ? FVB_OK : cuda_fail(e, "fvb_up_rhs");
}

fvb_status fvb_apply_bc(void *Qp, int n, int np, int bc_x, int bc_y, int layout, int dtype, void *stream)
{
    if (!Qp) return fail(FVB_ERR_INVALID, "null argument");
    if (np < n || (np - n) % 2 || bc_x < 0 || bc_x > 2 || bc_y < 0 || bc_y > 2 || (layout != 0 && layout != 1))
        return fail(FVB_ERR_INVALID, "bad geometry or boundary condition");
    BufView v{n, (np - n) / 2, np, 0, (long long)np * np};
    if (v.g > n) return fail(FVB_ERR_INVALID, "ghost width exceeds n");
    cudaError_t e = dtype == FVB_F64 ? bc_fill<double>((double *)Qp, v, bc_x, bc_y, (cudaStream_t)stream)
                                     : bc_fill<float>((float *)Qp, v, bc_x, bc_y, (cudaStream_t)stream);
    return e == cudaSuccess ? FVB_OK : cuda_fail(e, "fvb_apply_bc");
}

fvb_status fvb_rk3_stage(int stage, void *Uo, const void *U0, const void *Uk, const void *L, double dt, int n,
                         int np, double gamma, int dtype, void *stream)
{
    if (!Uo || !U0 || !L || (stage != 1 && !Uk)) return fail(FVB_ERR_INVALID, "null argument");
    if (stage < 1 || stage > 3 || np < n || (np - n) % 2) return fail(FVB_ERR_INVALID, "bad stage or geometry");
    int g = (np - n) / 2;
    cudaError_t e;
    if (dtype == FVB_F64)
        e = rk3_stage_ref<double>(stage, (double *)Uo, (const double *)U0, (const double *)Uk, (const double *)L, dt,
                                  n, np, g, gamma, (cudaStream_t)stream);
    else
        e = rk3_stage_ref<float>(stage, (float *)Uo, (const float *)U0, (const float *)Uk, (const float *)L,
                                 (float)dt, n, np, g, gamma, (cudaStream_t)stream);
    return e == cudaSuccess ? FVB_OK : cuda_fail(e, "fvb_rk3_stage");
}

fvb_status fvb_max(const void *x, size_t n, void *out_dev, int dtype, void *stream)
{
    if (!x || !out_dev) return fail(FVB_ERR_INVALID, "null argument");
    cudaError_t e = max_ref(x, n, out_dev, dtype, (cudaStream_t)stream);
    return e == cudaSuccess ? FVB_OK : cuda_fail(e, "fvb_max");
}

}  // extern "C"
