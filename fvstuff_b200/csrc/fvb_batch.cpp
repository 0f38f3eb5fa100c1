// fvb_batch.cpp -- the batched form: many grids of different sizes advanced
// together.  Every grid ("instance") keeps its own buffers, step control
// (dt, t, lam_max) and stop time on the device; a tile table maps each tile
// of every live instance to (instance slot, tile index), and one persistent
// launch of the stage kernel per RK stage walks that table.  The step (three
// launches, or six for the ping-pong FP32c state) is captured once as a CUDA
// graph whose arguments point at the table, so instances join and leave
// between replays without re-capturing.
#include <algorithm>
#include <cstring>
#include <vector>

#include "fvb_host.h"

using namespace fvb;

namespace {

struct Instance {
    int live = 0;        // slot in use
    int in_table = 0;    // its tiles are in the tile table
    int done = 0;        // reached t_end or failed, reported by poll
    int reported = 0;
    int home = 0;        // buffer parity holding its state once out of the table
    Geometry G{};
    void *block = nullptr;
    size_t bytes = 0;
    fvb_instance_desc desc{};
    GridDev gd{};
};

}  // namespace

struct fvb_batch {
    fvb_batch_config cfg{};
    int prec = P32C, order = 7, g = 4, internal = INT_CONS_HILO;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int max_inst = 4096;
    size_t budget = 0, in_use = 0;
    std::vector<Instance> inst;
    Ctrl *ctrl_dev = nullptr;       // [max_inst]
    Ctrl *ctrl_host = nullptr;      // pinned mirror
    GridDev *desc_dev = nullptr;    // [max_inst]
    GridDev *desc_host = nullptr;   // pinned staging
    TileRef *tiles_dev = nullptr;
    TileRef *tiles_host = nullptr;  // pinned staging
    int *ntiles_dev = nullptr;
    int *ntiles_host = nullptr;
    double *sums_dev = nullptr;     // per-block partials of fvb_batch_instance_sums
    double *sums_host = nullptr;    // pinned
    size_t tiles_cap = 0;
    int shape = 0;
    int ctas = 0;
    int parity = 0;
    int steps_per_graph = 1;
    bool dirty = true;
    bool use_graph = true;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    void *staging = nullptr;
    size_t staging_bytes = 0;
};

static void drop_graphs(fvb_batch *b)
{
    for (auto &g : b->gexec)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

static StageArgs batch_args(const fvb_batch *b, int stage, int parity)
{
    StageArgs a{};
    a.grids = b->desc_dev;
    a.ctrls = b->ctrl_dev;
    a.tiles = b->tiles_dev;
    a.ntiles = b->ntiles_dev;
    a.stage = stage;
    a.parity = parity;
    return a;
}

static cudaError_t launch_steps(fvb_batch *b, int nsteps)
{
    for (int k = 0; k < nsteps; ++k) {
        for (int stage = 1; stage <= 3; ++stage) {
            // (each grid's step control is evaluated inside the stage kernel)
            cudaError_t e = launch_stage(b->prec, b->order, b->shape, batch_args(b, stage, b->parity), b->ctas,
                                         b->stream);
            if (e != cudaSuccess) return e;
        }
        if (b->prec == P32C) b->parity ^= 1;
    }
    return cudaSuccess;
}

static cudaError_t capture(fvb_batch *b, int parity)
{
    int saved = b->parity;
    b->parity = parity;
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { b->parity = saved; return e; }
    cudaError_t el = launch_steps(b, b->steps_per_graph);
    e = cudaStreamEndCapture(b->stream, &graph);
    b->parity = saved;
    if (el != cudaSuccess) { if (graph) cudaGraphDestroy(graph); return el; }
    if (e != cudaSuccess) return e;
    e = cudaGraphInstantiate(&b->gexec[parity], graph, 0);
    cudaGraphDestroy(graph);
    return e;
}

// Rebuild the tile table from the live, unfinished instances and upload it
// (stream-ordered, so the next launch sees it).
static fvb_status upload_table(fvb_batch *b)
{
    const TileShape &ts = kTileShapes[b->shape];
    size_t total = 0;
    for (auto &I : b->inst)
        if (I.live && I.in_table) {
            int tx, nt;
            tile_dims(b->shape, I.G.n, tx, nt);
            total += nt;
        }
    if (total > b->tiles_cap) {
        size_t cap = std::max(total, b->tiles_cap * 2 + 1024);
        cudaStreamSynchronize(b->stream);
        if (b->tiles_dev) cudaFree(b->tiles_dev);
        if (b->tiles_host) cudaFreeHost(b->tiles_host);
        b->tiles_dev = nullptr;
        b->tiles_host = nullptr;
        cudaError_t e = cudaMalloc(&b->tiles_dev, cap * sizeof(TileRef));
        if (e == cudaSuccess) e = cudaMallocHost(&b->tiles_host, cap * sizeof(TileRef));
        if (e != cudaSuccess) return cuda_fail(e, "tile table");
        b->tiles_cap = cap;
        drop_graphs(b);  // the table moved
    }
    // the pinned staging buffers may still feed an earlier upload
    cudaError_t e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return cuda_fail(e, "sync");
    size_t k = 0;
    for (int slot = 0; slot < (int)b->inst.size(); ++slot) {
        Instance &I = b->inst[slot];
        if (!(I.live && I.in_table)) continue;
        int tx, nt;
        tile_dims(b->shape, I.G.n, tx, nt);
        I.gd.tiles_x = tx;
        b->desc_host[slot] = I.gd;
        for (int t = 0; t < nt; ++t) b->tiles_host[k++] = TileRef{slot, t};
    }
    (void)ts;
    *b->ntiles_host = (int)k;
    e = cudaMemcpyAsync(b->desc_dev, b->desc_host, sizeof(GridDev) * b->inst.size(), cudaMemcpyHostToDevice,
                        b->stream);
    if (e == cudaSuccess && k)
        e = cudaMemcpyAsync(b->tiles_dev, b->tiles_host, k * sizeof(TileRef), cudaMemcpyHostToDevice, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->ntiles_dev, b->ntiles_host, sizeof(int), cudaMemcpyHostToDevice, b->stream);
    if (e != cudaSuccess) return cuda_fail(e, "table upload");
    b->dirty = false;
    return FVB_OK;
}

static void *inst_state(const fvb_batch *b, const Instance &I, int parity)
{
    return I.gd.st[b->internal == INT_CONS_HILO ? parity : 0];
}

static int inst_parity(const fvb_batch *b, const Instance &I) { return I.in_table ? b->parity : I.home; }

extern "C" {

fvb_status fvb_batch_create(const fvb_batch_config *cfg, fvb_batch **out)
{
    if (!cfg || !out) return fail(FVB_ERR_INVALID, "null argument");
    *out = nullptr;
    if (cfg->precision != FVB_PREC_F32C && cfg->precision != FVB_PREC_F64)
        return fail(FVB_ERR_INVALID, "batched form runs FP32c or FP64");
    if (cfg->order != 7 && cfg->order != 0) return fail(FVB_ERR_INVALID, "batched form is built for UP7");
    if (cfg->tile >= kNumTileShapes) return fail(FVB_ERR_INVALID, "tile variant out of range");
    cudaError_t e = cudaSetDevice(cfg->device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
    fvb_batch *b = new fvb_batch();
    b->cfg = *cfg;
    b->prec = cfg->precision == FVB_PREC_F64 ? P64 : P32C;
    b->internal = prec_internal(cfg->precision);
    b->max_inst = cfg->max_instances > 0 ? cfg->max_instances : 4096;
    b->budget = cfg->hbm_budget ? cfg->hbm_budget : (size_t)150 << 30;
    b->use_graph = cfg->use_graph != 0;
    b->steps_per_graph = b->prec == P32C ? 2 : 1;
    b->inst.resize(b->max_inst);
    if (cfg->stream) b->stream = (cudaStream_t)cfg->stream;
    else {
        e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) { delete b; return cuda_fail(e, "stream"); }
        b->own_stream = true;
    }
    {
        // instances come and go: keep device memory they free in the
        // stream-ordered pool for the next one rather than returning it to the
        // driver at every synchronisation
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, cfg->device) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    e = cudaMalloc(&b->ctrl_dev, sizeof(Ctrl) * b->max_inst);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->ctrl_dev, 0, sizeof(Ctrl) * b->max_inst, b->stream);
    if (e == cudaSuccess) e = cudaMallocHost(&b->ctrl_host, sizeof(Ctrl) * b->max_inst);
    if (e == cudaSuccess) e = cudaMalloc(&b->desc_dev, sizeof(GridDev) * b->max_inst);
    if (e == cudaSuccess) e = cudaMallocHost(&b->desc_host, sizeof(GridDev) * b->max_inst);
    if (e == cudaSuccess) e = cudaMalloc(&b->ntiles_dev, sizeof(int));
    if (e == cudaSuccess) e = cudaMallocHost(&b->ntiles_host, sizeof(int));
    if (e != cudaSuccess) { fvb_batch_destroy(b); return cuda_fail(e, "batch allocation"); }
    std::memset(b->desc_host, 0, sizeof(GridDev) * b->max_inst);
    // a batched launch walks many tiles, as a large grid does: tune there
    b->shape = cfg->tile >= 0 ? cfg->tile : autotune_shape(b->prec, 7, 4096);
    int per_sm = stage_max_ctas_per_sm(b->prec, 7, b->shape);
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cfg->device);
    if (per_sm <= 0 || sms <= 0) { fvb_batch_destroy(b); return fail(FVB_ERR_CUDA, "stage kernel cannot launch"); }
    b->ctas = per_sm * sms;
    *out = b;
    return FVB_OK;
}

void fvb_batch_destroy(fvb_batch *b)
{
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graphs(b);
    for (auto &I : b->inst)
        if (I.block) cudaFree(I.block);
    cudaFree(b->ctrl_dev);
    cudaFreeHost(b->ctrl_host);
    cudaFree(b->desc_dev);
    cudaFreeHost(b->desc_host);
    cudaFree(b->tiles_dev);
    cudaFreeHost(b->tiles_host);
    cudaFree(b->ntiles_dev);
    cudaFreeHost(b->ntiles_host);
    if (b->staging) cudaFree(b->staging);
    if (b->sums_dev) cudaFree(b->sums_dev);
    if (b->sums_host) cudaFreeHost(b->sums_host);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

size_t fvb_batch_instance_bytes(const fvb_batch *b, int n)
{
    if (!b || n < 4) return 0;
    return (make_geometry(n, b->g, b->cfg.precision).bytes + 255) / 256 * 256 + TM_COUNT * sizeof(CUtensorMap);
}

int fvb_batch_active(const fvb_batch *b)
{
    if (!b) return 0;
    int k = 0;
    for (auto &I : b->inst) k += I.live && I.in_table;
    return k;
}

size_t fvb_batch_bytes_in_use(const fvb_batch *b) { return b ? b->in_use : 0; }

fvb_status fvb_batch_add(fvb_batch *b, const fvb_instance_desc *d, int *id)
{
    if (!b || !d || !id) return fail(FVB_ERR_INVALID, "null argument");
    if (d->n < b->g || d->n > 65536) return fail(FVB_ERR_INVALID, "n out of range");
    for (int bc : {d->bc_x, d->bc_y})
        if (bc < 0 || bc > 2) return fail(FVB_ERR_INVALID, "bad boundary condition");
    if (!(d->length > 0) || !(d->cfl > 0) || !(d->gamma > 1) || !(d->t_end > 0))
        return fail(FVB_ERR_INVALID, "length, cfl, t_end must be > 0 and gamma > 1");
    int slot = -1;
    for (int k = 0; k < b->max_inst; ++k)
        if (!b->inst[k].live) { slot = k; break; }
    if (slot < 0) return fail(FVB_ERR_NOMEM, "no free instance slot (max %d)", b->max_inst);
    Geometry G = make_geometry(d->n, b->g, b->cfg.precision);
    const size_t tmap_off = (G.bytes + 255) / 256 * 256;
    G.bytes = tmap_off + TM_COUNT * sizeof(CUtensorMap);
    if (b->in_use + G.bytes > b->budget)
        return fail(FVB_ERR_NOMEM, "HBM budget: %zu + %zu > %zu bytes", b->in_use, G.bytes, b->budget);
    Instance &I = b->inst[slot];
    I = Instance();
    cudaError_t e = cudaMallocAsync(&I.block, G.bytes, b->stream);
    if (e != cudaSuccess) return fail(FVB_ERR_NOMEM, "device allocation of %zu bytes: %s", G.bytes,
                                      cudaGetErrorString(e));
    e = cudaMemsetAsync(I.block, 0, G.bytes, b->stream);
    I.G = G;
    I.bytes = G.bytes;
    I.desc = *d;
    grid_pointers(I.gd, I.block, G, b->cfg.precision);
    I.gd.bcx = d->bc_x;
    I.gd.bcy = d->bc_y;
    I.gd.h = d->length / d->n;
    I.gd.gam = d->gamma;
    I.gd.ctrl = b->ctrl_dev + slot;
    I.gd.tmap = nullptr;
    {
        // descriptors for the batch's tile shape; every batched grid uses TMA
        int tx, nt;
        tile_dims(b->shape, d->n, tx, nt);
        I.gd.tiles_x = tx;
        CUtensorMap maps[TM_COUNT];
        if (!encode_tile_maps(I.gd, b->prec, 7, b->shape, maps)) {
            cudaFreeAsync(I.block, b->stream);
            I = Instance();
            return fail(FVB_ERR_CUDA, "cannot encode TMA descriptors for n = %d", d->n);
        }
        CUtensorMap *dm = (CUtensorMap *)((char *)I.block + tmap_off);
        if (e == cudaSuccess) e = put_tile_maps(maps, dm, b->stream);
        I.gd.tmap = dm;
    }
    // initial state: FP64 primitives on the device, imported into the buffer
    // the current parity reads
    size_t need = (size_t)4 * d->n * d->n * sizeof(double);
    if (need > b->staging_bytes) {
        if (b->staging) cudaFreeAsync(b->staging, b->stream);
        b->staging = nullptr;
        e = cudaMallocAsync(&b->staging, need, b->stream);
        if (e != cudaSuccess) { cudaFreeAsync(I.block, b->stream); I = Instance(); return cuda_fail(e, "staging"); }
        b->staging_bytes = need;
    }
    int p = b->parity;
    BufView v = view_of(I.gd);
    if (e == cudaSuccess) e = init_case_prim64((double *)b->staging, d->n, d->x0, d->y0, I.gd.h, d->gamma, d->ic,
                                               b->stream);
    ExtView ev{1, b->g, G.np, FVB_LAYOUT_PRIM, FVB_F64};
    if (e == cudaSuccess)
        e = import_state(b->staging, ev, inst_state(b, I, p), I.gd.lo[p], v, b->internal, d->gamma, b->stream);
    if (e == cudaSuccess) {
        if (b->internal == INT_PRIM64) e = bc_fill<double>((double *)I.gd.st[0], v, d->bc_x, d->bc_y, b->stream);
        else {
            e = bc_fill<float>((float *)I.gd.st[p], v, d->bc_x, d->bc_y, b->stream);
            if (e == cudaSuccess) e = bc_fill<float>((float *)I.gd.lo[p], v, d->bc_x, d->bc_y, b->stream);
        }
    }
    if (e == cudaSuccess) e = lam_into(inst_state(b, I, p), v, b->internal, d->gamma, &I.gd.ctrl->lam_acc, b->stream);
    if (e == cudaSuccess) e = ctrl_set(I.gd.ctrl, d->t_end, 1, 0.0, d->cfl, I.gd.h, b->stream);
    if (e != cudaSuccess) {
        cudaFreeAsync(I.block, b->stream);
        I = Instance();
        return cuda_fail(e, "instance set-up");
    }
    I.live = 1;
    I.in_table = 1;
    b->in_use += G.bytes;
    b->dirty = true;
    *id = slot;
    return FVB_OK;
}

fvb_status fvb_batch_run(fvb_batch *b, int nsteps)
{
    NvtxRange nvtx_range("fvb_batch_run");
    if (!b || nsteps < 0) return fail(FVB_ERR_INVALID, "bad argument");
    if (b->dirty) {
        fvb_status st = upload_table(b);
        if (st) return st;
    }
    if (*b->ntiles_host == 0) return FVB_OK;
    cudaError_t e = cudaSuccess;
    if (b->use_graph) {
        while (nsteps >= b->steps_per_graph && e == cudaSuccess) {
            int p = b->parity;
            if (!b->gexec[p]) e = capture(b, p);
            if (e == cudaSuccess) e = cudaGraphLaunch(b->gexec[p], b->stream);
            nsteps -= b->steps_per_graph;
        }
    }
    if (e == cudaSuccess) e = launch_steps(b, nsteps);
    return e == cudaSuccess ? FVB_OK : cuda_fail(e, "batch step");
}

fvb_status fvb_batch_poll(fvb_batch *b, int *ids, int cap, int *n_done)
{
    NvtxRange nvtx_range("fvb_batch_poll");
    if (!b || !n_done) return fail(FVB_ERR_INVALID, "null argument");
    *n_done = 0;
    cudaError_t e = cudaMemcpyAsync(b->ctrl_host, b->ctrl_dev, sizeof(Ctrl) * b->max_inst, cudaMemcpyDeviceToHost,
                                    b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return cuda_fail(e, "poll");
    for (int slot = 0; slot < b->max_inst; ++slot) {
        Instance &I = b->inst[slot];
        if (!I.live) continue;
        const Ctrl &c = b->ctrl_host[slot];
        if (!I.done && (c.status != 0 || !(c.t < c.t_stop))) {
            I.done = 1;
            if (I.in_table) {
                I.in_table = 0;
                I.home = b->parity;
                b->dirty = true;
            }
        }
        if (I.done && !I.reported && *n_done < cap) {
            I.reported = 1;
            if (ids) ids[*n_done] = slot;
            ++*n_done;
        }
    }
    return FVB_OK;
}

fvb_status fvb_batch_get_state(fvb_batch *b, int id, void *dst, int layout, int dtype, int interior_only)
{
    if (!b || !dst) return fail(FVB_ERR_INVALID, "null argument");
    if (id < 0 || id >= b->max_inst || !b->inst[id].live) return fail(FVB_ERR_NOT_FOUND, "no instance %d", id);
    Instance &I = b->inst[id];
    int p = inst_parity(b, I);
    long long side = interior_only ? I.G.n : I.G.np;
    size_t bytes = (size_t)4 * side * side * (dtype == FVB_F64 ? 8 : 4);
    void *tmp = nullptr;
    cudaError_t e = cudaMallocAsync(&tmp, bytes, b->stream);
    ExtView ev{interior_only ? 1 : 0, b->g, I.G.np, layout, dtype};
    if (e == cudaSuccess)
        e = export_state(inst_state(b, I, p), I.gd.lo[p], view_of(I.gd), b->internal, tmp, ev, I.desc.gamma,
                         b->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst, tmp, bytes, cudaMemcpyDeviceToHost, b->stream);
    if (tmp) cudaFreeAsync(tmp, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    return e == cudaSuccess ? FVB_OK : cuda_fail(e, "batch state");
}

fvb_status fvb_batch_instance_stats(fvb_batch *b, int id, fvb_stats *st)
{
    if (!b || !st) return fail(FVB_ERR_INVALID, "null argument");
    if (id < 0 || id >= b->max_inst || !b->inst[id].live) return fail(FVB_ERR_NOT_FOUND, "no instance %d", id);
    Ctrl c;
    cudaError_t e = cudaMemcpyAsync(b->ctrl_host + id, b->ctrl_dev + id, sizeof(Ctrl), cudaMemcpyDeviceToHost,
                                    b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) return cuda_fail(e, "stats");
    c = b->ctrl_host[id];
    std::memset(st, 0, sizeof *st);
    st->t = c.t;
    st->dt = c.dt;
    std::memcpy(&st->lam_max, &c.lam_acc, sizeof(double));
    st->t_stop = c.t_stop;
    st->steps = c.step;
    st->status = c.status;
    return FVB_OK;
}

fvb_status fvb_batch_instance_sums(fvb_batch *b, int id, fvb_stats *st)
{
    if (!b || !st) return fail(FVB_ERR_INVALID, "null argument");
    if (id < 0 || id >= b->max_inst || !b->inst[id].live) return fail(FVB_ERR_NOT_FOUND, "no instance %d", id);
    constexpr int kBlocks = 592;
    cudaError_t e = cudaSuccess;
    if (!b->sums_dev) {
        e = cudaMalloc(&b->sums_dev, sizeof(double) * 5 * kBlocks);
        if (e == cudaSuccess) e = cudaMallocHost(&b->sums_host, sizeof(double) * 5 * kBlocks);
        if (e != cudaSuccess) return cuda_fail(e, "sums buffers");
    }
    Instance &I = b->inst[id];
    const int p = inst_parity(b, I);
    e = sums_partials(inst_state(b, I, p), I.gd.lo[p], view_of(I.gd), b->internal, I.desc.gamma, b->sums_dev,
                      kBlocks, b->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->sums_host, b->sums_dev, sizeof(double) * 5 * kBlocks, cudaMemcpyDeviceToHost,
                            b->stream);
    if (e != cudaSuccess) return cuda_fail(e, "sums");
    const fvb_status r = fvb_batch_instance_stats(b, id, st);  // waits for the stream
    if (r) return r;
    double acc[5] = {0, 0, 0, 0, 0};
    for (int k = 0; k < kBlocks; ++k)
        for (int q = 0; q < 5; ++q) acc[q] += b->sums_host[k * 5 + q];
    const double h2 = I.gd.h * I.gd.h;
    for (int q = 0; q < 4; ++q) st->sums[q] = acc[q] * h2;
    st->nonfinite = acc[4] > 0;
    return FVB_OK;
}

fvb_status fvb_batch_remove(fvb_batch *b, int id)
{
    if (!b) return fail(FVB_ERR_INVALID, "null argument");
    if (id < 0 || id >= b->max_inst || !b->inst[id].live) return fail(FVB_ERR_NOT_FOUND, "no instance %d", id);
    Instance &I = b->inst[id];
    if (I.in_table) b->dirty = true;
    if (b->dirty) {
        // the table must stop naming the slot before its memory is released
        I.in_table = 0;
        fvb_status st = upload_table(b);
        if (st) return st;
    }
    cudaFreeAsync(I.block, b->stream);
    // a zero step control is inactive: the stage-control kernel leaves it be
    cudaError_t e = cudaMemsetAsync(b->ctrl_dev + id, 0, sizeof(Ctrl), b->stream);
    b->in_use -= I.bytes;
    I = Instance();
    return e == cudaSuccess ? FVB_OK : cuda_fail(e, "step control reset");
}

}  // extern "C"
