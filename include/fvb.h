/*
 * fvb.h -- C ABI of libfvb, a B200-native (sm_100a) implementation of the
 * finite-volume Euler time step of fvStuff's fv_up7_ducros_2d.cu (UP7
 * reconstruction, Ducros-blended HLLC/HLLE flux, SSP-RK3, CFL max-wavespeed
 * reduction) and keep_fv_euler_2d.cu (ECKEP + JST/MOVERS-RH flux).
 *
 * Plain C types only: pointers, sizes, enums.  Every entry point returns an
 * fvb_status and never exits the process; fvb_last_error() gives the text.
 *
 * State layout ("IDX_P", fv_up7_ducros_2d.cu:49-56, keep_fv_euler_2d.cu:79-80):
 * padded SoA of 4 variables, element (q, jp, ip) at q*Np*Np + jp*Np + ip,
 * Np = N + 2g, interior cell (j, i) at (jp, ip) = (j + g, i + g), j = row (y),
 * i = column (x).  g = (order + 1) / 2 for the UP path (4 for UP7) and 2 for
 * KEEP.  Variables are primitives [rho, u, v, p] (FVB_LAYOUT_PRIM, what
 * fv_up7 stores) or conserved [rho, rho u, rho v, E] (FVB_LAYOUT_CONS, what
 * keep_fv stores); either can be read or written in any precision mode.
 */
#ifndef FVB_H
#define FVB_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define FVB_API __attribute__((visibility("default")))
#else
#define FVB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fvb_status {
    FVB_OK = 0,
    FVB_ERR_INVALID = 1,      /* bad argument or configuration            */
    FVB_ERR_CUDA = 2,         /* a CUDA call failed                        */
    FVB_ERR_NOMEM = 3,        /* device allocation or HBM budget exceeded  */
    FVB_ERR_BLOWUP = 4,       /* lam_max not > 0 (fv_up7_ducros_2d.cu:997) */
    FVB_ERR_DT_UNDERFLOW = 5, /* dt < 1e-14 (fv_up7_ducros_2d.cu:1002)     */
    FVB_ERR_NOT_FOUND = 6,    /* unknown batch instance id                 */
    FVB_ERR_TIMEOUT = 7       /* a bounded wait gave up                    */
} fvb_status;

typedef enum fvb_flux {
    FVB_FLUX_UP_DUCROS = 0,   /* UP-order recon + Ducros HLLC/HLLE (fv_up7_ducros_2d.cu:370-507) */
    FVB_FLUX_KEEP = 1,        /* ECKEP + JST/MOVERS-RH (keep_fv_euler_2d.cu:298-369)              */
    /* UP7 + Ducros blend with carb_fv's alternatives to HLLC on the
     * reconstructed states (carb_fv_2d.cu:116-211; FP64, order 7) */
    FVB_FLUX_UP_DUCROS_HLL = 2,
    FVB_FLUX_UP_DUCROS_ROE = 3,
    /* rec3 (kappa = 1/3) reconstruction of the conserved variables, face
     * Zhang-Shu scaling, HLLC, 2x2-block Zhang-Shu positivity limiter after
     * every stage (fv_rec3_2d.cu:147-353; FP64, periodic, N even) */
    FVB_FLUX_REC3 = 4,
    /* the scheme kept in fv_up7_ducros_2d.cu.bak: UP-order reconstruction of
     * the conserved variables, HLLC, and a D2 artificial viscosity gated by
     * a Ducros weight from the 6th-order velocity divergence
     * (fv_up7_ducros_2d.cu.bak:287-390; FP64, order 3, 5, 7 or 9, ghost width
     * max((order + 1) / 2, 3); coefficients from fvb_set_d2av) */
    FVB_FLUX_UP_HLLC_D2AV = 5
} fvb_flux;

typedef enum fvb_precision {
    FVB_PREC_F64 = 0,         /* the plain method in FP64 (the reference retyped to double)     */
    FVB_PREC_F32 = 1,         /* FP32 as shipped: FP32 state, FP64 reconstruction arithmetic    */
    FVB_PREC_F32C = 2         /* FP32 flux/divergence, compensated hi/lo FP32 conserved state   */
} fvb_precision;

typedef enum fvb_bc {
    FVB_BC_REFLECT = 0,       /* reflecting walls (fv_up7_ducros_2d.cu:338-362)   */
    FVB_BC_PERIODIC = 1,      /* periodic (keep_fv_euler_2d.cu:224-243)           */
    FVB_BC_TRANSMISSIVE = 2   /* zero-gradient copy of the nearest interior cell  */
} fvb_bc;

typedef enum fvb_layout {
    FVB_LAYOUT_PRIM = 0,      /* [rho, u, v, p]      */
    FVB_LAYOUT_CONS = 1       /* [rho, rho u, rho v, E] */
} fvb_layout;

typedef enum fvb_dtype { FVB_F32 = 0, FVB_F64 = 1 } fvb_dtype;

typedef enum fvb_where { FVB_HOST = 0, FVB_DEVICE = 1 } fvb_where;

typedef enum fvb_case_kind {
    FVB_CASE_SOD = 0,         /* circular Sod, tanh-smoothed (fv_up7_ducros_2d.cu:618-639)        */
    FVB_CASE_VORTEX = 1,      /* isentropic vortex with mean flow (rt_dg_euler_2d.cu:1334-1356)   */
    FVB_CASE_KH = 2,          /* Kelvin-Helmholtz double shear layer with seeded noise            */
    FVB_CASE_RIEMANN4 = 3,    /* four-quadrant 2-D Riemann problem from a seed                    */
    FVB_CASE_KEEP_SOD = 4,    /* keep_fv circular Sod (keep_fv_euler_2d.cu:448-469)               */
    FVB_CASE_LMV = 5,         /* stationary low-Mach vortex (keep_fv_euler_2d.cu:471-513)         */
    FVB_CASE_UNIFORM = 6,     /* constant state (param[0..3] = rho, u, v, p)                      */
    /* fv_rec3_2d.cu's cases, as conserved cell averages (FVB_FLUX_REC3 only,
     * fv_rec3_2d.cu:383-416): sharp circular Sod 10/0.125, the paper's
     * isentropic vortex on [0,10]^2, the Gresho vortex (param[0] = eps) */
    FVB_CASE_REC3_SOD = 7,
    FVB_CASE_PAPER_VORTEX = 8,
    FVB_CASE_GRESHO = 9
} fvb_case_kind;

/* One grid: N x N cells on [x0, x0 + length] x [y0, y0 + length], h = length / N. */
typedef struct fvb_config {
    int n;                    /* cells per side (>= g)                            */
    int order;                /* UP order: 3, 5, 7 or 9 (ignored by KEEP)         */
    int flux;                 /* fvb_flux                                         */
    int precision;            /* fvb_precision                                    */
    int bc_x, bc_y;           /* fvb_bc on the x and y boundaries                 */
    double x0, y0, length;    /* domain                                           */
    double gamma;             /* ratio of specific heats (1.4 in the reference)   */
    double cfl;               /* dt = cfl * h / lam_max                           */
    int device;               /* CUDA device ordinal                              */
    void *stream;             /* cudaStream_t to run on, NULL = a private stream  */
    int tile;                 /* stage-kernel tile variant, -1 = autotuned        */
} fvb_config;

typedef struct fvb_case {
    int kind;                 /* fvb_case_kind                                    */
    uint64_t seed;            /* KH noise / Riemann quadrant states               */
    double param[8];          /* case parameters; see fvb_case_default          */
} fvb_case;

typedef struct fvb_stats {
    double t;                 /* simulated time                                   */
    double dt;                /* last step's dt                                   */
    double lam_max;           /* max |u|+|v|+c of the current state               */
    double t_stop;            /* current stop time                                */
    int64_t steps;            /* steps taken                                      */
    int status;               /* fvb_status of the device-side step control       */
    int nonfinite;            /* 1 if a non-finite cell was seen by the last sums */
    double sums[4];           /* FP64 sums of rho, rho u, rho v, E times h^2 (fvb_stats_sums only) */
} fvb_stats;

typedef struct fvb_solver fvb_solver;

FVB_API const char *fvb_version(void);
/* name of CUDA device `device` (valid until the next call on this thread),
 * or NULL with the error set       the "Device" line, fv_up7_ducros_2d.cu:894-898 */
FVB_API const char *fvb_device_name(int device);
/* text of the last error on this thread */
FVB_API const char *fvb_last_error(void);
/* default configuration: UP7 + Ducros, FP64, reflecting walls, [0,1]^2,
 * gamma 1.4, CFL 0.4 -- the settings of fv_up7_ducros_2d.cu:889 */
FVB_API void fvb_config_default(fvb_config *cfg, int n);

/* default parameters of a test case on [x0, x0+length] x [y0, y0+length]:
 *   SOD      param = {xc, yc, radius, rho_out, rho_in, p_out, p_in}
 *                    = centre, 0.25 length, 0.125, 11, 0.1, 10 (fv_up7_ducros_2d.cu:629-637)
 *   VORTEX   param = {beta, u0, v0, xc, yc} = 5, 1, 1, centre
 *   KH       param = {yc, half width, rho_in, rho_out, u_in, u_out, p, noise}
 *                    = centre, 0.25 length, 2, 1, -0.5, 0.5, 2.5, 1e-3; seed 12345
 *   RIEMANN4 param = {xm, ym} = centre; quadrant states drawn from `seed`
 *   LMV      param = {eps} = 0.1
 *   UNIFORM  param = {rho, u, v, p} = 1, 0, 0, 1                             */
FVB_API void fvb_case_default(fvb_case *c, int kind, double x0, double y0, double length);

/* Solver lifetime; replaces the allocations of fv_up7_ducros_2d.cu:904-919. */
FVB_API fvb_status fvb_create(const fvb_config *cfg, fvb_solver **out);
FVB_API void fvb_destroy(fvb_solver *s);
FVB_API int fvb_ghost_width(const fvb_solver *s);

/* Initial state on the device, ghosts filled, t = 0
 * (fv_up7_ducros_2d.cu:973-976 ic_kernel + apply_bc). */
FVB_API fvb_status fvb_init_case(fvb_solver *s, const fvb_case *c);

/* Write / read the full padded IDX_P array (4 x Np x Np) or, with
 * interior_only, the (4 x N x N) interior.  set_state refills the ghosts,
 * recomputes lam_max and resets t = 0. */
FVB_API fvb_status fvb_set_state(fvb_solver *s, const void *src, int layout, int dtype, int where, int interior_only);
FVB_API fvb_status fvb_get_state(fvb_solver *s, void *dst, int layout, int dtype, int where, int interior_only);
/* hi/lo words of the compensated state, conserved, interior, FP32 each */
FVB_API fvb_status fvb_get_state_hilo(fvb_solver *s, float *hi, float *lo);

/* Frame fields of fv_up7's composite image (fv_up7_ducros_2d.cu:800-829,
 * :511-526), extracted on the device from the state as it stands after the
 * steps already enqueued: density, 6th-order vorticity (4th-order for the
 * two-ghost-layer KEEP and rec3 families), the Ducros cell sensor (for
 * FVB_FLUX_UP_HLLC_D2AV its velocity-divergence weight), |v| and pressure,
 * 5 planes of N x N floats (row-major, j = 0 at the
 * bottom).  fvb_frame_begin enqueues the extraction on the solver's stream and
 * the copy to host on a second stream, and returns; steps enqueued after it
 * run while the frame is copied and written.  fvb_frame_end waits for that
 * copy and writes the 5 N N floats to `out`.  The reference computes these on
 * the host after a blocking copy of the whole state. */
FVB_API fvb_status fvb_frame_begin(fvb_solver *s);
FVB_API fvb_status fvb_frame_end(fvb_solver *s, float *out);

/* Checkpoint / resume: the exact internal state (every padded buffer word),
 * the time, the step count and the wave-speed max that sets the next dt, so
 * a resumed run continues bit for bit.  The reference writes images only
 * (fv_up7_ducros_2d.cu:757-881) and cannot resume.  load requires a solver
 * created with the same n, flux, order and precision. */
FVB_API fvb_status fvb_save(fvb_solver *s, const char *path);
FVB_API fvb_status fvb_load(fvb_solver *s, const char *path);

/* Enqueue up to nsteps SSP-RK3 steps on the solver's stream without waiting.
 * Each step picks dt = cfl h / lam_max, clamped so t lands on t_stop; steps
 * at t >= t_stop do nothing.  Replaces the loop body of
 * fv_up7_ducros_2d.cu:995-1032 (one fused kernel per RK stage). */
FVB_API fvb_status fvb_step(fvb_solver *s, int nsteps, double t_stop);
/* Run until t >= t_stop (or max_steps), synchronising every `chunk` steps. */
FVB_API fvb_status fvb_advance(fvb_solver *s, double t_stop, int64_t max_steps, int chunk);
/* Wait for the stream and read the step control (t, dt, lam_max, status). */
FVB_API fvb_status fvb_sync(fvb_solver *s, fvb_stats *st);
/* The same read without waiting for later work: fvb_stats_post enqueues a
 * copy of the step control, as it stands after the steps enqueued so far,
 * into slot `slot` (0 .. FVB_STATS_SLOTS-1) of a pinned ring;
 * fvb_stats_wait waits for that copy only and fills st.  A caller can post
 * after each fvb_step and wait for the previous step's slot while the next
 * step runs.  A slot is reused by its next post. */
#define FVB_STATS_SLOTS 8
FVB_API fvb_status fvb_stats_post(fvb_solver *s, int slot);
FVB_API fvb_status fvb_stats_wait(fvb_solver *s, int slot, fvb_stats *st);

/* The rec3 family's count of 2x2 blocks whose mean itself needed the floor
 * fix (the "brutal mean-fix activations" fv_rec3_2d.cu:250, :594 reports),
 * since the state was last set; 0 for the other flux families.  Waits for
 * the solver's stream. */
FVB_API fvb_status fvb_limiter_fixes(fvb_solver *s, int64_t *count);

/* Coefficients of the FVB_FLUX_UP_HLLC_D2AV viscosity: C2 (Ducros-gated),
 * Cg (global, weight 1 - S_D) and the sensor's sound-speed scale sc; the
 * .bak's command-line arguments 2-4, defaults 0.5, 0, 0.05
 * (fv_up7_ducros_2d.cu.bak:742-744).  FVB_ERR_INVALID for other fluxes. */
FVB_API fvb_status fvb_set_d2av(fvb_solver *s, double c2, double cg, double sc);

/* Failure injection for tests (no counterpart in the reference): the next
 * stage launch of this solver issues no first halo-box load on its first
 * CTA, so that CTA's bounded wait (one second of GPU time) runs out, the
 * kernel ends normally and the solver's status becomes FVB_ERR_TIMEOUT --
 * the path a lost asynchronous copy would take.  The GPU context stays
 * usable; the solver stops stepping, as after a blow-up. */
FVB_API fvb_status fvb_debug_drop_load(fvb_solver *s);
/* As fvb_sync, plus FP64 conserved sums over the interior. */
FVB_API fvb_status fvb_stats_sums(fvb_solver *s, fvb_stats *st);
/* Record the whole step (three stage kernels) as a CUDA graph and replay it
 * from fvb_step; on by default for grids of 512^2 cells or fewer. */
FVB_API fvb_status fvb_set_graph(fvb_solver *s, int enable);

/* ---- the reference's kernel-level contract, on caller device buffers in
 * the IDX_P layout (Np arbitrary >= N + 2g), async on `stream` ---------- */

/* residual -(dF/dx + dG/dy) of the conserved variables (4 x N x N, unpadded)
 * and lam = |u|+|v|+c (N x N) of a padded primitive state (UP path)
 *                                          replaces compute_rhs, fv_up7_ducros_2d.cu:370-374 */
FVB_API fvb_status fvb_up_rhs(const void *Qp, void *rhs, void *lam, int n, int np, int order, double h,
                      double gamma, int dtype, void *stream);
/* fill the ghost ring of a padded state   replaces apply_bc, fv_up7_ducros_2d.cu:338-339 */
FVB_API fvb_status fvb_apply_bc(void *Qp, int n, int np, int bc_x, int bc_y, int layout, int dtype, void *stream);
/* one SSP-RK3 stage on primitives (stage 1: U0 + dt L; 2: 3/4 U0 + 1/4 (Uk + dt L);
 * 3: 1/3 U0 + 2/3 (Uk + dt L)), floors rho, p >= 1e-14
 *                                          replaces rk3_s1/s2/s3, fv_up7_ducros_2d.cu:531-590 */
FVB_API fvb_status fvb_rk3_stage(int stage, void *Uo, const void *U0, const void *Uk, const void *L,
                         double dt, int n, int np, double gamma, int dtype, void *stream);
/* max over n values, from 0 (NaN skipped), written to a device scalar
 *                                          replaces reduce_max/gpu_max, fv_up7_ducros_2d.cu:593-612 */
FVB_API fvb_status fvb_max(const void *x, size_t n, void *out_dev, int dtype, void *stream);

/* Up to nsteps SSP-RK3 steps (UP7 + Ducros, FP64) of a caller-held padded
 * primitive state Qp (device, IDX_P layout, n <= 512, n + 8 <= np <= 520),
 * starting at time t0 and stopping at t_stop, WITHOUT allocating device
 * memory: for callers that cannot call cudaMalloc, e.g. an application whose
 * device memory belongs to its own pool allocator or is fixed at start-up.
 * The stage buffers and step control live in one fixed __device__ array of
 * the library (about 17 MB, held on every GPU that loads libfvb.so), so
 * calls that overlap on the GPU race with each other.  The ghost ring of Qp
 * is refilled.  Every call looks up the array's address in the current
 * context (the first one on a device may also load the library's kernels);
 * make that first call before any stream capture on that device.  When st
 * is non-null the call waits for the stream and fills it; st->steps counts
 * the steps of this call only (fvb_stats of a solver counts from its
 * creation), st->t is the time reached from t0.  No counterpart in the
 * reference. */
FVB_API fvb_status fvb_step_noalloc(double *Qp, int n, int np, double h, double cfl, double gamma, int bc_x,
                                    int bc_y, int nsteps, double t0, double t_stop, void *stream, fvb_stats *st);

/* ---- batched form: many uneven grids in one persistent launch per stage -- */

typedef struct fvb_batch_config {
    int precision;            /* FVB_PREC_F32C (default) or FVB_PREC_F64           */
    int order;                /* 7                                                 */
    int device;
    void *stream;
    size_t hbm_budget;        /* bytes of state the batch may hold (0 = 150 GB)    */
    int max_instances;        /* 0 = 4096                                          */
    int use_graph;            /* capture the three stages as a CUDA graph          */
    int tile;                 /* stage-kernel tile variant, -1 = autotuned         */
} fvb_batch_config;

typedef struct fvb_instance_desc {
    int n;
    int bc_x, bc_y;
    double x0, y0, length;
    double gamma, cfl;
    double t_end;             /* the instance finishes at t_end                    */
    fvb_case ic;              /* initial state                                     */
} fvb_instance_desc;

typedef struct fvb_batch fvb_batch;

FVB_API fvb_status fvb_batch_create(const fvb_batch_config *cfg, fvb_batch **out);
FVB_API void fvb_batch_destroy(fvb_batch *b);
/* device bytes one instance of this size needs in this batch */
FVB_API size_t fvb_batch_instance_bytes(const fvb_batch *b, int n);
/* admit an instance (FVB_ERR_NOMEM when it would exceed the HBM budget);
 * it joins the tile table at the next fvb_batch_run */
FVB_API fvb_status fvb_batch_add(fvb_batch *b, const fvb_instance_desc *d, int *id);
/* enqueue nsteps steps of every active instance (3 persistent launches per step) */
FVB_API fvb_status fvb_batch_run(fvb_batch *b, int nsteps);
/* wait, then list instances that reached t_end (or failed) since the last poll */
FVB_API fvb_status fvb_batch_poll(fvb_batch *b, int *ids, int cap, int *n_done);
FVB_API fvb_status fvb_batch_get_state(fvb_batch *b, int id, void *dst, int layout, int dtype, int interior_only);
FVB_API fvb_status fvb_batch_instance_stats(fvb_batch *b, int id, fvb_stats *st);
/* as fvb_batch_instance_stats, plus the instance's FP64 conserved sums and
 * its non-finite flag (what fvb_stats_sums gives for a solver) */
FVB_API fvb_status fvb_batch_instance_sums(fvb_batch *b, int id, fvb_stats *st);
FVB_API fvb_status fvb_batch_remove(fvb_batch *b, int id);
FVB_API int fvb_batch_active(const fvb_batch *b);
FVB_API size_t fvb_batch_bytes_in_use(const fvb_batch *b);

/* ---- serving loop: continuous batching of a request stream ------------ */

typedef struct fvb_request {
    double arrival;           /* seconds after the start of the run                */
    fvb_instance_desc desc;
    void *out;                /* host buffer for the final interior state (4 x n x n
                               * in out_layout / out_dtype), written before the
                               * instance retires; NULL = keep no result          */
    int out_layout;           /* FVB_LAYOUT_PRIM or FVB_LAYOUT_CONS                */
    int out_dtype;            /* FVB_F64 or FVB_F32                                */
} fvb_request;

typedef struct fvb_request_result {
    double admitted;          /* seconds after start when it joined the batch      */
    double finished;          /* seconds after start when its result was ready     */
    int status;               /* fvb_status of the instance                        */
    int64_t steps;
    double t;
} fvb_request_result;

enum {
    FVB_SERVE_FIFO = 0,           /* admit in arrival order                          */
    FVB_SERVE_SHORTEST_FIRST = 1  /* admit the waiting request of least estimated
                                   * work first (n^3 t_end: cells x steps)           */
};

typedef struct fvb_serve_config {
    fvb_batch_config batch;
    int steps_per_round;      /* steps per batch round between admissions (0 = 8) */
    int policy;               /* FVB_SERVE_FIFO or FVB_SERVE_SHORTEST_FIRST        */
    double max_cells;         /* admit while the live instances hold fewer interior
                               * cells than this (0 = no limit but HBM and slots);
                               * one instance is always admitted                   */
    double max_seconds;       /* give up after this long (0 = no limit)            */
} fvb_serve_config;

/* Play the request stream in real time: requests become visible at their
 * arrival time, are admitted (in the policy's order; a request that does not
 * fit blocks the ones behind it) as HBM budget, slots and the cell cap allow,
 * advance together, and are retired when they reach t_end, their final state
 * copied to reqs[i].out first.  Blocks until all are done.  res[i] matches
 * reqs[i]. */
FVB_API fvb_status fvb_serve_run(const fvb_serve_config *cfg, const fvb_request *reqs, int nreq,
                         fvb_request_result *res, double *wall_seconds);

#ifdef __cplusplus
}
#endif
#endif /* FVB_H */
