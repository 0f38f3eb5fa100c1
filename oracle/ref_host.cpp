/*
 * ref_host.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Host build of the reference solvers' own kernels (the extracted source is
 * generated by oracle/build.py into oracle/_ref/ from the read-only
 * reference checkout and never committed).  This file only adds the launch
 * emulation and the host time loop around those kernels; it is compiled
 * three ways:
 *   -DREF_UP7 -DREF_REAL=float   fv_up7_ducros_2d.cu as shipped
 *   -DREF_UP7 -DREF_REAL=double  its float->double retype
 *   -DREF_KEEP                   keep_fv_euler_2d.cu (FP64 already)
 *   -DREF_CARB -DUSE_DOUBLE      carb_fv_2d.cu's Riemann solvers, FP64
 *   -DREF_REC3 -Dreal=double -Dreall=double   fv_rec3_2d.cu, FP64
 *   -DREF_BAK                    fv_up7_ducros_2d.cu.bak (FP64 already)
 * Used to pin the oracle restatement bit-for-bit and as the CPU baseline
 * ("kind": "reference") of bench.py.
 */
#include "ref_shim.h"
#include <omp.h>

thread_local ref_dim3 blockIdx, threadIdx, blockDim, gridDim;

#include REF_INC

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)

static int g_nthreads = 0;  /* 0: OpenMP default */

/* One call of `body` per virtual block b in [0, n): blockDim = 1 and
 * gridDim = n, so the kernel's grid-stride loop runs exactly once, for
 * work item b.  Blocks are split over threads in contiguous chunks.     */
template <class F>
static void grid_launch(long long n, F &&body)
{
    int nt = g_nthreads > 0 ? g_nthreads : omp_get_max_threads();
#pragma omp parallel num_threads(nt)
    {
        threadIdx = { 0, 0, 0 };
        blockDim = { 1, 1, 1 };
        gridDim = { (unsigned)n, 1, 1 };
#pragma omp for schedule(static)
        for (long long b = 0; b < n; ++b) {
            blockIdx = { (unsigned)b, 0, 0 };
            body();
        }
    }
}

template <class R>
static R host_max(const R *x, long long n)
{
    R m = 0;
    for (long long k = 0; k < n; ++k) m = std::fmax(m, x[k]);
    return m;
}

/* Ghost fills the shipped UP7 solver does not have, composed for the
 * harness: periodic as keep_fv_euler_2d.cu:224-243 and zero-gradient
 * (nearest interior cell) as carb_fv_2d.cu:245-247, applied on every side. */
template <class R>
static void harness_bc(R *Q, int N, int Np, int bc)
{
    int g = (Np - N) / 2;
    long long Np2 = (long long)Np * Np;
    int nt = g_nthreads > 0 ? g_nthreads : omp_get_max_threads();
    /* rows in parallel; an interior row only has its 2g ghost columns */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int jp = 0; jp < Np; ++jp)
        for (int ip = 0; ip < Np; ++ip) {
            bool gx = ip < g || ip >= N + g, gy = jp < g || jp >= N + g;
            if (!gx && !gy) {
                ip = N + g - 1;
                continue;
            }
            int ir = ip, jr = jp;
            if (bc == 1) {
                if (ip < g) ir = ip + N; else if (ip >= N + g) ir = ip - N;
                if (jp < g) jr = jp + N; else if (jp >= N + g) jr = jp - N;
            } else {
                if (ip < g) ir = g; else if (ip >= N + g) ir = N + g - 1;
                if (jp < g) jr = g; else if (jp >= N + g) jr = N + g - 1;
            }
            for (int q = 0; q < 4; ++q) Q[q * Np2 + (long long)jp * Np + ip] = Q[q * Np2 + (long long)jr * Np + ir];
        }
}

extern "C" void ref_set_threads(int n) { g_nthreads = n; }
extern "C" int ref_get_threads(void) { return g_nthreads > 0 ? g_nthreads : omp_get_max_threads(); }

#if defined(REF_UP7)
typedef REF_REAL R;
#define API(n) CAT(n, REF_SFX)

extern "C" {

int API(ref_up7_order_)(void) { return ORDER; }

void API(ref_up7_rhs_)(const R *Qp, R *RHS, R *lam, int N, int Np, R h)
{
    grid_launch((long long)N * N, [&] { compute_rhs(Qp, RHS, lam, N, Np, h); });
}

void API(ref_up7_bc_)(R *Qp, int N, int Np, int bc)
{
    if (bc == 0) grid_launch((long long)Np * Np, [&] { apply_bc(Qp, N, Np); });
    else harness_bc(Qp, N, Np, bc);
}

void API(ref_up7_rk3_)(int stage, R *Uo, const R *U0, const R *Uk, const R *L, R dt, int N, int Np)
{
    long long n = (long long)N * N;
    if (stage == 1) grid_launch(n, [&] { rk3_s1(Uo, U0, L, dt, N, Np); });
    else if (stage == 2) grid_launch(n, [&] { rk3_s2(Uo, U0, Uk, L, dt, N, Np); });
    else grid_launch(n, [&] { rk3_s3(Uo, U0, Uk, L, dt, N, Np); });
}

/* single faces with a general normal (fv_up7_ducros_2d.cu:237-328, :149-186) */
void API(ref_up7_hllc_)(const R *WL, const R *WR, R nx, R ny, R *F) { hllc_n(WL, WR, nx, ny, F); }
void API(ref_up7_hlle_)(const R *WL, const R *WR, R nx, R ny, R *F) { hlle_n(WL, WR, nx, ny, F); }
void API(ref_up7_up7_)(const R *s, R *vL, R *vR) { up7(s, vL, vR); }
void API(ref_up7_ducros_)(const R *P, int Np, int jp, int ip, R *sx, R *sy)
{
    *sx = ducros_x_p(P, jp, ip, Np);
    *sy = ducros_y_p(P, jp, ip, Np);
}

void API(ref_up7_ic_sod_)(R *U, int N, int Np, R h)
{
    grid_launch((long long)N * N, [&] { ic_kernel(U, N, Np, h); });
}

/* the time loop of fv_up7_ducros_2d.cu:990-1032 around the kernels above,
 * stopping at max_steps or t >= t_stop (the frame-clamped dt lands on it) */
int API(ref_up7_run_)(R *U, int N, R h, R cfl, int bc, int max_steps, double t_stop, double *info)
{
    const int g = ORDER_G;
    int Np = N + 2 * g;
    size_t nP = (size_t)4 * Np * Np, n1 = (size_t)N * N;
    R *U0 = (R *)malloc(sizeof(R) * nP), *U1 = (R *)malloc(sizeof(R) * nP);
    R *U2 = (R *)malloc(sizeof(R) * nP), *L = (R *)malloc(sizeof(R) * 4 * n1);
    R *lam = (R *)malloc(sizeof(R) * n1);
    memcpy(U1, U, sizeof(R) * nP);
    memcpy(U2, U, sizeof(R) * nP);
    API(ref_up7_rhs_)(U, L, lam, N, Np, h);
    R lmax = host_max(lam, (long long)n1), t = 0, dt = 0, ts = (R)t_stop;
    int step = 0, status = 0;
    while (step < max_steps && t < ts) {
        if (!(lmax > (R)0)) { status = 1; break; }
        dt = cfl * h / lmax;
        if (t + dt > ts) dt = ts - t;
        if (dt < (R)1e-14) { status = 2; break; }
        memcpy(U0, U, sizeof(R) * nP);
        API(ref_up7_rk3_)(1, U1, U0, U0, L, dt, N, Np);
        API(ref_up7_bc_)(U1, N, Np, bc);
        API(ref_up7_rhs_)(U1, L, lam, N, Np, h);
        API(ref_up7_rk3_)(2, U2, U0, U1, L, dt, N, Np);
        API(ref_up7_bc_)(U2, N, Np, bc);
        API(ref_up7_rhs_)(U2, L, lam, N, Np, h);
        API(ref_up7_rk3_)(3, U, U0, U2, L, dt, N, Np);
        API(ref_up7_bc_)(U, N, Np, bc);
        API(ref_up7_rhs_)(U, L, lam, N, Np, h);
        lmax = host_max(lam, (long long)n1);
        t += dt;
        step++;
    }
    if (info) { info[0] = (double)t; info[1] = step; info[2] = (double)lmax; info[3] = (double)dt; }
    free(U0); free(U1); free(U2); free(L); free(lam);
    return status;
}

}  /* extern "C" */

#elif defined(REF_CARB)
/* carb_fv_2d.cu's Riemann solvers (real = double with -DUSE_DOUBLE) */

extern "C" {
void ref_carb_hllc(const real *WL, const real *WR, real nx, real ny, real *F) { hllc_n(WL, WR, nx, ny, F); }
void ref_carb_hll(const real *WL, const real *WR, real nx, real ny, real *F) { hll_n(WL, WR, nx, ny, F); }
void ref_carb_roe(const real *WL, const real *WR, real nx, real ny, real *F) { roe_n(WL, WR, nx, ny, F); }
}  /* extern "C" */

#elif defined(REF_REC3)
/* fv_rec3_2d.cu built with real = reall = double */
typedef double R;

extern "C" {

void ref_rec3_rhs(const R *Qp, R *RHS, R *lam, int N, int Np, R h)
{
    std::memset(RHS, 0, sizeof(R) * 4 * (size_t)N * N);
    grid_launch((long long)N * N, [&] { compute_rhs(Qp, RHS, lam, N, Np, h); });
}
int ref_rec3_limit(R *Qp, int N, int Np)
{
    g_brutal_count = 0;
    grid_launch((long long)(N / 2) * (N / 2), [&] { limit_positivity_blocks(Qp, N, Np); });
    return g_brutal_count;
}
void ref_rec3_bc(R *Qp, int N, int Np) { grid_launch((long long)Np * Np, [&] { apply_bc(Qp, N, Np); }); }
void ref_rec3_ic(R *Qp, int N, int Np, R h, int icase, R p0)
{
    std::memset(Qp, 0, sizeof(R) * 4 * (size_t)Np * Np);
    grid_launch((long long)N * N, [&] { ic_kernel(Qp, N, Np, h, icase, p0); });
}
void ref_rec3_hllc(const R *WL, const R *WR, R nx, R ny, R *F) { hllc_n(WL, WR, nx, ny, F); }
void ref_rec3_scale(const R *Ub, R *U) { scale_to_admissible(Ub, U); }

/* the time loop of fv_rec3_2d.cu:551-590 around the kernels above, on a
 * state that has had its limiter pass and ghost fill */
int ref_rec3_run(R *U, int N, R h, R cfl, int max_steps, double t_stop, double *info)
{
    int Np = N + 2 * G_GHOST;
    size_t nP = (size_t)4 * Np * Np, n1 = (size_t)N * N;
    R *U0 = (R *)malloc(sizeof(R) * nP), *U1 = (R *)malloc(sizeof(R) * nP);
    R *L = (R *)malloc(sizeof(R) * 4 * n1), *lam = (R *)malloc(sizeof(R) * n1);
    std::memcpy(U1, U, sizeof(R) * nP);
    ref_rec3_rhs(U, L, lam, N, Np, h);
    R lmax = host_max(lam, (long long)n1), t = 0, dt = 0;
    int step = 0, status = 0, brutal = 0;
    while (step < max_steps && t < (R)t_stop) {
        if (!(lmax > 0.)) { status = 1; break; }
        dt = cfl * h / lmax;
        if (t + dt > (R)t_stop) dt = (R)t_stop - t;
        if (dt < 1e-14) { status = 2; break; }
        std::memcpy(U0, U, sizeof(R) * nP);
        grid_launch((long long)n1, [&] { rk_stage(U1, U0, U0, L, 0., 1., 0., dt, N, Np); });
        brutal += ref_rec3_limit(U1, N, Np);
        ref_rec3_bc(U1, N, Np);
        ref_rec3_rhs(U1, L, lam, N, Np, h);
        grid_launch((long long)n1, [&] { rk_stage(U1, U0, U1, L, 0.75, 0.25, 0., dt, N, Np); });
        brutal += ref_rec3_limit(U1, N, Np);
        ref_rec3_bc(U1, N, Np);
        ref_rec3_rhs(U1, L, lam, N, Np, h);
        grid_launch((long long)n1, [&] { rk_stage(U, U0, U1, L, (R)(1. / 3.), (R)(2. / 3.), 0., dt, N, Np); });
        brutal += ref_rec3_limit(U, N, Np);
        ref_rec3_bc(U, N, Np);
        ref_rec3_rhs(U, L, lam, N, Np, h);
        lmax = host_max(lam, (long long)n1);
        t += dt;
        step++;
    }
    if (info) { info[0] = t; info[1] = step; info[2] = lmax; info[3] = dt; info[4] = brutal; }
    free(U0); free(U1); free(L); free(lam);
    return status;
}

}  /* extern "C" */

#elif defined(REF_BAK)
/* fv_up7_ducros_2d.cu.bak: unpadded N x N conserved state read through its
 * reflecting fetch */
typedef double R;

extern "C" {

void ref_bak_rhs(const R *U, R *RHS, R *lam, int N, R h, R C2, R Cg, R sc, int order)
{
    grid_launch((long long)N * N, [&] { compute_rhs(U, RHS, lam, N, h, C2, Cg, sc, order); });
}
void ref_bak_sensor(const R *U, R *SD, int N, R h, R sc)
{
    grid_launch((long long)N * N, [&] { compute_sensor(U, SD, N, h, sc); });
}
void ref_bak_rk3(int stage, R *Uo, const R *U0, const R *Uk, const R *L, R dt, int N)
{
    int M = 4 * N * N;
    if (stage == 1) grid_launch(M, [&] { rk3_s1(Uo, U0, L, dt, M); });
    else if (stage == 2) grid_launch(M, [&] { rk3_s2(Uo, U0, Uk, L, dt, M); });
    else grid_launch(M, [&] { rk3_s3(Uo, U0, Uk, L, dt, M); });
}
void ref_bak_ic(R *U, int N, R h) { grid_launch((long long)N * N, [&] { ic_kernel(U, N, h); }); }
void ref_bak_hllc(const R *UL, const R *UR, int yface, R *F)
{
    if (yface) hllc_y(UL, UR, F);
    else hllc_x(UL, UR, F);
}

/* the time loop of fv_up7_ducros_2d.cu.bak:848-872 (residual and lam at
 * the start of a step, dt = CFL h / lam_max clamped onto t_stop, stop on
 * dt < 1e-14), with the stop on a non-positive lam_max of this library */
int ref_bak_run(R *U, int N, R h, R cfl, R C2, R Cg, R sc, int order, int max_steps, double t_stop, double *info)
{
    size_t n4 = (size_t)4 * N * N, n1 = (size_t)N * N;
    R *U0 = (R *)malloc(sizeof(R) * n4), *U1 = (R *)malloc(sizeof(R) * n4);
    R *U2 = (R *)malloc(sizeof(R) * n4), *L = (R *)malloc(sizeof(R) * n4), *lam = (R *)malloc(sizeof(R) * n1);
    ref_bak_rhs(U, L, lam, N, h, C2, Cg, sc, order);
    R lmax = host_max(lam, (long long)n1), t = 0, dt = 0;
    int step = 0, status = 0;
    while (step < max_steps && t < t_stop) {
        if (!(lmax > 0.)) { status = 1; break; }
        dt = cfl * h / lmax;
        if (t + dt > t_stop) dt = t_stop - t;
        if (dt < 1e-14) { status = 2; break; }
        memcpy(U0, U, sizeof(R) * n4);
        ref_bak_rk3(1, U1, U0, U0, L, dt, N);
        ref_bak_rhs(U1, L, lam, N, h, C2, Cg, sc, order);
        ref_bak_rk3(2, U2, U0, U1, L, dt, N);
        ref_bak_rhs(U2, L, lam, N, h, C2, Cg, sc, order);
        ref_bak_rk3(3, U, U0, U2, L, dt, N);
        ref_bak_rhs(U, L, lam, N, h, C2, Cg, sc, order);
        lmax = host_max(lam, (long long)n1);
        t += dt;
        step++;
    }
    if (info) { info[0] = t; info[1] = step; info[2] = lmax; info[3] = dt; }
    free(U0); free(U1); free(U2); free(L); free(lam);
    return status;
}

}  /* extern "C" */

#elif defined(REF_KEEP)
typedef double R;

extern "C" {

void ref_keep_ed(const R *Qp, R *ed, int N, int Np)
{
    grid_launch((long long)N * N, [&] { compute_ed(Qp, ed, N, Np); });
}

void ref_keep_rhs(const R *Qp, R *RHS, R *lam, int N, int Np, R h, R edmax)
{
    grid_launch((long long)N * N, [&] { compute_rhs(Qp, RHS, lam, N, Np, h, edmax); });
}

void ref_keep_rk(R *Uo, const R *Ua, const R *Ub, const R *L, R ca, R cb, R cl, R dt, int N, int Np)
{
    grid_launch((long long)N * N, [&] { rk_stage(Uo, Ua, Ub, L, ca, cb, cl, dt, N, Np); });
}

void ref_keep_bc(R *Qp, int N, int Np)
{
    grid_launch((long long)Np * Np, [&] { apply_bc(Qp, N, Np); });
}

void ref_keep_ic(R *Qp, int N, int Np, R h, int lmv, R eps)
{
    if (lmv) grid_launch((long long)N * N, [&] { ic_lmv(Qp, N, Np, h, eps); });
    else grid_launch((long long)N * N, [&] { ic_sod(Qp, N, Np, h); });
}

void ref_keep_err_lmv(const R *Qp, R *erho, R *ep, int N, int Np, R h, R eps)
{
    grid_launch((long long)N * N, [&] { err_lmv(Qp, erho, ep, N, Np, h, eps); });
}

static void rhs_of(const R *U, R *L, R *lam, R *ed, int N, int Np, R h)
{
    ref_keep_ed(U, ed, N, Np);
    R edm = host_max(ed, (long long)N * N);
    ref_keep_rhs(U, L, lam, N, Np, h, edm);
}

/* the time loop of keep_fv_euler_2d.cu:691-725 around the kernels above */
int ref_keep_run(R *U, int N, R h, R cfl, int max_steps, double t_stop, double *info)
{
    const int g = G_GHOST;
    int Np = N + 2 * g;
    size_t nP = (size_t)4 * Np * Np, n1 = (size_t)N * N;
    R *U0 = (R *)malloc(sizeof(R) * nP), *U1 = (R *)malloc(sizeof(R) * nP);
    R *U2 = (R *)malloc(sizeof(R) * nP), *L = (R *)malloc(sizeof(R) * 4 * n1);
    R *lam = (R *)malloc(sizeof(R) * n1), *ed = (R *)malloc(sizeof(R) * n1);
    memcpy(U1, U, sizeof(R) * nP);
    memcpy(U2, U, sizeof(R) * nP);
    rhs_of(U, L, lam, ed, N, Np, h);
    R lmax = host_max(lam, (long long)n1), t = 0, dt = 0;
    int step = 0, status = 0;
    while (step < max_steps && t < t_stop) {
        if (!(lmax > 0.)) { status = 1; break; }
        dt = cfl * h / lmax;
        if (t + dt > t_stop) dt = t_stop - t;
        if (dt < 1e-14) { status = 2; break; }
        memcpy(U0, U, sizeof(R) * nP);
        ref_keep_rk(U1, U0, U0, L, 1., 0., 1., dt, N, Np);
        ref_keep_bc(U1, N, Np);
        rhs_of(U1, L, lam, ed, N, Np, h);
        ref_keep_rk(U2, U0, U1, L, 0.75, 0.25, 0.25, dt, N, Np);
        ref_keep_bc(U2, N, Np);
        rhs_of(U2, L, lam, ed, N, Np, h);
        ref_keep_rk(U, U0, U2, L, 1. / 3., 2. / 3., 2. / 3., dt, N, Np);
        ref_keep_bc(U, N, Np);
        rhs_of(U, L, lam, ed, N, Np, h);
        lmax = host_max(lam, (long long)n1);
        t += dt;
        step++;
    }
    if (info) { info[0] = t; info[1] = step; info[2] = lmax; info[3] = dt; }
    free(U0); free(U1); free(U2); free(L); free(lam); free(ed);
    return status;
}

}  /* extern "C" */
#endif
