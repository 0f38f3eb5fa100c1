/*
 * ref_gpu.cu -- TEST INFRASTRUCTURE ONLY.
 *
 * GPU build of the reference solvers' own CUDA kernels: the reference
 * source file itself is #included (REF_CU; the FP64 variant is the
 * float->double retype generated by oracle/build.py under oracle/_ref/),
 * with its main() renamed (and exported as refg_main).  This file adds host-array entry
 * points that run the reference's kernels with the reference's launch
 * configuration and host loop, for the GPU parity tests and for timing the
 * reference kernels on the same device.
 */
#define main fvref_unused_main
#include REF_CU
#undef main

/* the reference program itself: its main() unchanged (argument parsing,
 * time loop, stdout lines and output files in the current directory), for
 * the tests that compare the command-line drivers' outputs with it */
extern "C" int refg_main(int argc, char **argv) { return fvref_unused_main(argc, argv); }

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)

/* periodic (keep_fv_euler_2d.cu:224-243) and zero-gradient
 * (carb_fv_2d.cu:245-247) ghost fills composed for the harness, launched
 * like the reference's own apply_bc */
template <class R>
__global__ void harness_bc_kernel(R *Q, int N, int Np, int bc)
{
    int g = (Np - N) / 2;
    long long Np2 = (long long)Np * Np;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < Np2;
         k += (long long)blockDim.x * gridDim.x) {
        int jp = (int)(k / Np), ip = (int)(k % Np);
        bool gx = ip < g || ip >= N + g, gy = jp < g || jp >= N + g;
        if (!gx && !gy) continue;
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

#define RET_ON_ERR(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) return (int)_e; } while (0)

#if defined(REF_UP7)
typedef REF_REAL R;
#define API(n) CAT(n, REF_SFX)

static void bc_launch(R *d, int N, int Np, int bc)
{
    if (bc == 0) apply_bc<<<GS_NBLK, BLOCK1D>>>(d, N, Np);
    else harness_bc_kernel<R><<<GS_NBLK, BLOCK1D>>>(d, N, Np, bc);
}

extern "C" {

/* the reference's frame of a padded primitive state Qh (host): its
 * compute_sensor and compute_derived kernels, the colour ranges of its
 * WRITE_FRAME (density 0.125 .. 10.1, vorticity symmetric about its largest
 * magnitude, sensor 0 .. 1, |v| 0 .. its max) and its write_ppm_2x2
 * (fv_up7_ducros_2d.cu:931-971, :835-881), into file `fn` */
int API(refg_up7_frame_)(const R *Qh, int N, R h, const char *fn)
{
    const int Np = N + 2 * ORDER_G;
    size_t nP = (size_t)4 * Np * Np, n1 = (size_t)N * N;
    R *dQ = nullptr, *dSD = nullptr, *dW = nullptr, *dV = nullptr;
    RET_ON_ERR(cudaMalloc(&dQ, nP * sizeof(R)));
    RET_ON_ERR(cudaMalloc(&dSD, n1 * sizeof(R)));
    RET_ON_ERR(cudaMalloc(&dW, n1 * sizeof(R)));
    RET_ON_ERR(cudaMalloc(&dV, n1 * sizeof(R)));
    RET_ON_ERR(cudaMemcpy(dQ, Qh, nP * sizeof(R), cudaMemcpyHostToDevice));
    compute_sensor<<<GS_NBLK, BLOCK1D>>>(dQ, dSD, N, Np);
    compute_derived<<<GS_NBLK, BLOCK1D>>>(dQ, dW, dV, N, Np, h);
    RET_ON_ERR(cudaDeviceSynchronize());
    R *rho = (R *)malloc(n1 * sizeof(R)), *sd = (R *)malloc(n1 * sizeof(R));
    R *vort = (R *)malloc(n1 * sizeof(R)), *vmag = (R *)malloc(n1 * sizeof(R));
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) rho[(size_t)j * N + i] = Qh[(size_t)(j + ORDER_G) * Np + i + ORDER_G];
    RET_ON_ERR(cudaMemcpy(sd, dSD, n1 * sizeof(R), cudaMemcpyDeviceToHost));
    RET_ON_ERR(cudaMemcpy(vort, dW, n1 * sizeof(R), cudaMemcpyDeviceToHost));
    RET_ON_ERR(cudaMemcpy(vmag, dV, n1 * sizeof(R), cudaMemcpyDeviceToHost));
    const R RHO_MIN = 0.125, RHO_MAX = 10.1;
    R wmax = 1e-10f, vmax = 1e-10f;
    for (size_t k = 0; k < n1; k++) {
        R aw = vort[k] < 0.0 ? -vort[k] : vort[k];
        if (aw > wmax) wmax = aw;
        if (vmag[k] > vmax) vmax = vmag[k];
    }
    write_ppm_2x2(fn, rho, RHO_MIN, RHO_MAX, 0, vort, -wmax, wmax, 3, sd, 0.0, 1.0, 2, vmag, 0.0, vmax, 1, N);
    free(rho); free(sd); free(vort); free(vmag);
    cudaFree(dQ); cudaFree(dSD); cudaFree(dW); cudaFree(dV);
    return 0;
}

/* one compute_rhs launch (fv_up7_ducros_2d.cu:370) on host arrays */
int API(refg_up7_rhs_)(const R *Qh, R *RHSh, R *lamh, int N, int Np, R h)
{
    size_t nP = (size_t)4 * Np * Np, n1 = (size_t)N * N;
    R *dQ = nullptr, *dR = nullptr, *dl = nullptr;
    RET_ON_ERR(cudaMalloc(&dQ, nP * sizeof(R)));
    RET_ON_ERR(cudaMalloc(&dR, 4 * n1 * sizeof(R)));
    RET_ON_ERR(cudaMalloc(&dl, n1 * sizeof(R)));
    RET_ON_ERR(cudaMemcpy(dQ, Qh, nP * sizeof(R), cudaMemcpyHostToDevice));
    compute_rhs<<<GS_NBLK, BLOCK1D>>>(dQ, dR, dl, N, Np, h);
    RET_ON_ERR(cudaGetLastError());
    RET_ON_ERR(cudaMemcpy(RHSh, dR, 4 * n1 * sizeof(R), cudaMemcpyDeviceToHost));
    RET_ON_ERR(cudaMemcpy(lamh, dl, n1 * sizeof(R), cudaMemcpyDeviceToHost));
    cudaFree(dQ); cudaFree(dR); cudaFree(dl);
    return 0;
}

/* the time loop of fv_up7_ducros_2d.cu:990-1032 on the device, with the
 * reference's kernels, launches, D2D copy and per-step gpu_max; ms_out gets
 * the CUDA-event time of the stepping loop (prologue excluded) */
int API(refg_up7_run_)(R *Uh, int N, R h, R cfl, int bc, int max_steps, double t_stop,
                       double *info, float *ms_out)
{
    const int g = ORDER_G;
    int Np = N + 2 * g;
    size_t sz4p = (size_t)4 * Np * Np * sizeof(R), n1 = (size_t)N * N;
    R *dU, *dU0, *dU1, *dU2, *dRHS, *dlam, *dtmp;
    RET_ON_ERR(cudaMalloc(&dU, sz4p)); RET_ON_ERR(cudaMalloc(&dU0, sz4p));
    RET_ON_ERR(cudaMalloc(&dU1, sz4p)); RET_ON_ERR(cudaMalloc(&dU2, sz4p));
    RET_ON_ERR(cudaMalloc(&dRHS, 4 * n1 * sizeof(R)));
    RET_ON_ERR(cudaMalloc(&dlam, n1 * sizeof(R)));
    RET_ON_ERR(cudaMalloc(&dtmp, GS_NBLK * sizeof(R)));
    RET_ON_ERR(cudaMemcpy(dU, Uh, sz4p, cudaMemcpyHostToDevice));
    RET_ON_ERR(cudaMemcpy(dU1, Uh, sz4p, cudaMemcpyHostToDevice));
    RET_ON_ERR(cudaMemcpy(dU2, Uh, sz4p, cudaMemcpyHostToDevice));
    compute_rhs<<<GS_NBLK, BLOCK1D>>>(dU, dRHS, dlam, N, Np, h);
    RET_ON_ERR(cudaDeviceSynchronize());
    R lmax = gpu_max(dlam, dtmp, (int)n1), t = 0, dt = 0, ts = (R)t_stop;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    cudaEventRecord(e0);
    int step = 0, status = 0;
    while (step < max_steps && t < ts) {
        if (!(lmax > (R)0)) { status = 1; break; }
        dt = cfl * h / lmax;
        if (t + dt > ts) dt = ts - t;
        if (dt < (R)1e-14) { status = 2; break; }
        RET_ON_ERR(cudaMemcpy(dU0, dU, sz4p, cudaMemcpyDeviceToDevice));
        rk3_s1<<<GS_NBLK, BLOCK1D>>>(dU1, dU0, dRHS, dt, N, Np);
        bc_launch(dU1, N, Np, bc);
        compute_rhs<<<GS_NBLK, BLOCK1D>>>(dU1, dRHS, dlam, N, Np, h);
        rk3_s2<<<GS_NBLK, BLOCK1D>>>(dU2, dU0, dU1, dRHS, dt, N, Np);
        bc_launch(dU2, N, Np, bc);
        compute_rhs<<<GS_NBLK, BLOCK1D>>>(dU2, dRHS, dlam, N, Np, h);
        rk3_s3<<<GS_NBLK, BLOCK1D>>>(dU, dU0, dU2, dRHS, dt, N, Np);
        bc_launch(dU, N, Np, bc);
        compute_rhs<<<GS_NBLK, BLOCK1D>>>(dU, dRHS, dlam, N, Np, h);
        lmax = gpu_max(dlam, dtmp, (int)n1);
        t += dt;
        step++;
    }
    cudaEventRecord(e1);
    RET_ON_ERR(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms_out) *ms_out = ms;
    RET_ON_ERR(cudaGetLastError());
    RET_ON_ERR(cudaMemcpy(Uh, dU, sz4p, cudaMemcpyDeviceToHost));
    if (info) { info[0] = (double)t; info[1] = step; info[2] = (double)lmax; info[3] = (double)dt; }
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    cudaFree(dU); cudaFree(dU0); cudaFree(dU1); cudaFree(dU2);
    cudaFree(dRHS); cudaFree(dlam); cudaFree(dtmp);
    return status ? -status : 0;
}

}  /* extern "C" */

#elif defined(REF_KEEP)
typedef double R;

extern "C" {

/* the reference's PNG frame of a padded conserved state Qh (host, g = 2):
 * its extract_fields kernel, the ranges of its WRITE_FRAME (left panel 0 ..
 * max(gpu_max, 1e-12), right panel the pressure's min .. max) and its
 * write_png_2panel (keep_fv_euler_2d.cu:541-589, :671-681), into file `fn` */
int refg_keep_frame(const double *Qh, int N, int lmv, const char *fn)
{
    const int Np = N + 2 * G_GHOST;
    size_t nP = (size_t)4 * Np * Np, n1 = (size_t)N * N;
    double *dQ = nullptr, *dl = nullptr, *dr = nullptr, *dt = nullptr;
    RET_ON_ERR(cudaMalloc(&dQ, nP * sizeof(double)));
    RET_ON_ERR(cudaMalloc(&dl, n1 * sizeof(double)));
    RET_ON_ERR(cudaMalloc(&dr, n1 * sizeof(double)));
    RET_ON_ERR(cudaMalloc(&dt, GS_NBLK * sizeof(double)));
    RET_ON_ERR(cudaMemcpy(dQ, Qh, nP * sizeof(double), cudaMemcpyHostToDevice));
    extract_fields<<<GS_NBLK, BLOCK1D>>>(dQ, dl, dr, N, Np, lmv);
    RET_ON_ERR(cudaDeviceSynchronize());
    double Lhi = gpu_max(dl, dt, N * N);
    double *hl = (double *)malloc(n1 * sizeof(double)), *hr = (double *)malloc(n1 * sizeof(double));
    RET_ON_ERR(cudaMemcpy(hl, dl, n1 * sizeof(double), cudaMemcpyDeviceToHost));
    RET_ON_ERR(cudaMemcpy(hr, dr, n1 * sizeof(double), cudaMemcpyDeviceToHost));
    double Rlo = 1e30, Rhi = -1e30;
    for (size_t q = 0; q < n1; q++) { Rlo = fmin(Rlo, hr[q]); Rhi = fmax(Rhi, hr[q]); }
    write_png_2panel(fn, hl, 0., fmax(Lhi, 1e-12), hr, Rlo, Rhi, N);
    free(hl); free(hr);
    cudaFree(dQ); cudaFree(dl); cudaFree(dr); cudaFree(dt);
    return 0;
}


/* compute_ed + gpu_max + compute_rhs (keep_fv_euler_2d.cu:640-645) on host arrays */
int refg_keep_rhs(const R *Qh, R *RHSh, R *lamh, int N, int Np, R h, R *edmax_out)
{
    size_t nP = (size_t)4 * Np * Np, n1 = (size_t)N * N;
    R *dQ, *dR, *dl, *de, *dt;
    RET_ON_ERR(cudaMalloc(&dQ, nP * sizeof(R)));
    RET_ON_ERR(cudaMalloc(&dR, 4 * n1 * sizeof(R)));
    RET_ON_ERR(cudaMalloc(&dl, n1 * sizeof(R)));
    RET_ON_ERR(cudaMalloc(&de, n1 * sizeof(R)));
    RET_ON_ERR(cudaMalloc(&dt, GS_NBLK * sizeof(R)));
    RET_ON_ERR(cudaMemcpy(dQ, Qh, nP * sizeof(R), cudaMemcpyHostToDevice));
    compute_ed<<<GS_NBLK, BLOCK1D>>>(dQ, de, N, Np);
    R edm = gpu_max(de, dt, (int)n1);
    compute_rhs<<<GS_NBLK, BLOCK1D>>>(dQ, dR, dl, N, Np, h, edm);
    RET_ON_ERR(cudaGetLastError());
    RET_ON_ERR(cudaMemcpy(RHSh, dR, 4 * n1 * sizeof(R), cudaMemcpyDeviceToHost));
    RET_ON_ERR(cudaMemcpy(lamh, dl, n1 * sizeof(R), cudaMemcpyDeviceToHost));
    if (edmax_out) *edmax_out = edm;
    cudaFree(dQ); cudaFree(dR); cudaFree(dl); cudaFree(de); cudaFree(dt);
    return 0;
}

/* the time loop of keep_fv_euler_2d.cu:691-725 with the reference kernels */
int refg_keep_run(R *Uh, int N, R h, R cfl, int max_steps, double t_stop, double *info, float *ms_out)
{
    const int g = G_GHOST;
    int Np = N + 2 * g;
    size_t szp = (size_t)4 * Np * Np * sizeof(R), n1 = (size_t)N * N, szc = 4 * n1 * sizeof(R);
    R *dU, *dU0, *dU1, *dU2, *dRHS, *dlam, *ded, *dtmp;
    RET_ON_ERR(cudaMalloc(&dU, szp)); RET_ON_ERR(cudaMalloc(&dU0, szp));
    RET_ON_ERR(cudaMalloc(&dU1, szp)); RET_ON_ERR(cudaMalloc(&dU2, szp));
    RET_ON_ERR(cudaMalloc(&dRHS, szc));
    RET_ON_ERR(cudaMalloc(&dlam, n1 * sizeof(R)));
    RET_ON_ERR(cudaMalloc(&ded, n1 * sizeof(R)));
    RET_ON_ERR(cudaMalloc(&dtmp, GS_NBLK * sizeof(R)));
    RET_ON_ERR(cudaMemcpy(dU, Uh, szp, cudaMemcpyHostToDevice));
    RET_ON_ERR(cudaMemcpy(dU1, Uh, szp, cudaMemcpyHostToDevice));
    RET_ON_ERR(cudaMemcpy(dU2, Uh, szp, cudaMemcpyHostToDevice));
    auto rhs_of = [&](R *U) {
        compute_ed<<<GS_NBLK, BLOCK1D>>>(U, ded, N, Np);
        R edm = gpu_max(ded, dtmp, (int)n1);
        cudaMemset(dRHS, 0, szc);
        compute_rhs<<<GS_NBLK, BLOCK1D>>>(U, dRHS, dlam, N, Np, h, edm);
    };
    rhs_of(dU);
    RET_ON_ERR(cudaDeviceSynchronize());
    R lmax = gpu_max(dlam, dtmp, (int)n1), t = 0, dt = 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    cudaEventRecord(e0);
    int step = 0, status = 0;
    while (step < max_steps && t < t_stop) {
        if (!(lmax > 0.)) { status = 1; break; }
        dt = cfl * h / lmax;
        if (t + dt > t_stop) dt = t_stop - t;
        if (dt < 1e-14) { status = 2; break; }
        RET_ON_ERR(cudaMemcpy(dU0, dU, szp, cudaMemcpyDeviceToDevice));
        rk_stage<<<GS_NBLK, BLOCK1D>>>(dU1, dU0, dU0, dRHS, 1., 0., 1., dt, N, Np);
        apply_bc<<<GS_NBLK, BLOCK1D>>>(dU1, N, Np);
        rhs_of(dU1);
        rk_stage<<<GS_NBLK, BLOCK1D>>>(dU2, dU0, dU1, dRHS, 0.75, 0.25, 0.25, dt, N, Np);
        apply_bc<<<GS_NBLK, BLOCK1D>>>(dU2, N, Np);
        rhs_of(dU2);
        rk_stage<<<GS_NBLK, BLOCK1D>>>(dU, dU0, dU2, dRHS, 1. / 3., 2. / 3., 2. / 3., dt, N, Np);
        apply_bc<<<GS_NBLK, BLOCK1D>>>(dU, N, Np);
        rhs_of(dU);
        lmax = gpu_max(dlam, dtmp, (int)n1);
        t += dt;
        step++;
    }
    cudaEventRecord(e1);
    RET_ON_ERR(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms_out) *ms_out = ms;
    RET_ON_ERR(cudaGetLastError());
    RET_ON_ERR(cudaMemcpy(Uh, dU, szp, cudaMemcpyDeviceToHost));
    if (info) { info[0] = t; info[1] = step; info[2] = lmax; info[3] = dt; }
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    cudaFree(dU); cudaFree(dU0); cudaFree(dU1); cudaFree(dU2);
    cudaFree(dRHS); cudaFree(dlam); cudaFree(ded); cudaFree(dtmp);
    return status ? -status : 0;
}

}  /* extern "C" */

#elif defined(REF_BAK)
typedef double R;

extern "C" {

/* the time loop of fv_up7_ducros_2d.cu.bak:848-872 with its kernels and
 * launches (unpadded N x N conserved state, reflecting fetch), stopping at
 * max_steps or t_stop; ms_out: CUDA-event time of the stepping loop */
int refg_bak_run(R *Uh, int N, R h, R cfl, R C2, R Cg, R sc, int order, int max_steps, double t_stop,
                 double *info, float *ms_out)
{
    size_t sz4 = (size_t)4 * N * N * sizeof(R), n1 = (size_t)N * N;
    int M = 4 * N * N;
    R *dU, *dU0, *dU1, *dU2, *dRHS, *dlam, *dtmp;
    RET_ON_ERR(cudaMalloc(&dU, sz4)); RET_ON_ERR(cudaMalloc(&dU0, sz4));
    RET_ON_ERR(cudaMalloc(&dU1, sz4)); RET_ON_ERR(cudaMalloc(&dU2, sz4));
    RET_ON_ERR(cudaMalloc(&dRHS, sz4));
    RET_ON_ERR(cudaMalloc(&dlam, n1 * sizeof(R)));
    RET_ON_ERR(cudaMalloc(&dtmp, GS_NBLK * sizeof(R)));
    RET_ON_ERR(cudaMemcpy(dU, Uh, sz4, cudaMemcpyHostToDevice));
    RET_ON_ERR(cudaDeviceSynchronize());
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    cudaEventRecord(e0);
    R t = 0, dt = 0, lmax = 0;
    int step = 0, status = 0;
    while (step < max_steps && t < t_stop) {
        compute_rhs<<<GS_NBLK, BLOCK1D>>>(dU, dRHS, dlam, N, h, C2, Cg, sc, order);
        lmax = gpu_max(dlam, dtmp, N * N);
        if (!(lmax > 0.)) { status = 1; break; }
        dt = cfl * h / lmax;
        if (t + dt > t_stop) dt = t_stop - t;
        if (dt < 1e-14) { status = 2; break; }
        RET_ON_ERR(cudaMemcpy(dU0, dU, sz4, cudaMemcpyDeviceToDevice));
        rk3_s1<<<GS_NBLK, BLOCK1D>>>(dU1, dU0, dRHS, dt, M);
        compute_rhs<<<GS_NBLK, BLOCK1D>>>(dU1, dRHS, dlam, N, h, C2, Cg, sc, order);
        rk3_s2<<<GS_NBLK, BLOCK1D>>>(dU2, dU0, dU1, dRHS, dt, M);
        compute_rhs<<<GS_NBLK, BLOCK1D>>>(dU2, dRHS, dlam, N, h, C2, Cg, sc, order);
        rk3_s3<<<GS_NBLK, BLOCK1D>>>(dU, dU0, dU2, dRHS, dt, M);
        t += dt;
        step++;
    }
    cudaEventRecord(e1);
    RET_ON_ERR(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms_out) *ms_out = ms;
    RET_ON_ERR(cudaGetLastError());
    RET_ON_ERR(cudaMemcpy(Uh, dU, sz4, cudaMemcpyDeviceToHost));
    if (info) { info[0] = t; info[1] = step; info[2] = lmax; info[3] = dt; }
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    cudaFree(dU); cudaFree(dU0); cudaFree(dU1); cudaFree(dU2);
    cudaFree(dRHS); cudaFree(dlam); cudaFree(dtmp);
    return status ? -status : 0;
}

}  /* extern "C" */

#elif defined(REF_REC3)
/* fv_rec3_2d.cu built with real = reall = double */
typedef double R;

extern "C" {

/* the time loop of fv_rec3_2d.cu:551-590 with its kernels and launches
 * (memset + atomicAdd-scatter compute_rhs, rk_stage, the 2x2-block limiter,
 * apply_bc, gpu_max) on a padded conserved state that has had its limiter
 * pass and ghost fill; ms_out: CUDA-event time of the stepping loop */
int refg_rec3_run(R *Uh, int N, R h, R cfl, int max_steps, double t_stop, double *info, float *ms_out)
{
    int Np = N + 2 * G_GHOST;
    size_t szP = (size_t)NVAR * Np * Np * sizeof(R), szC = (size_t)NVAR * N * N * sizeof(R);
    R *dU, *dU0, *dU1, *dRHS, *dlam, *dtmp;
    RET_ON_ERR(cudaMalloc(&dU, szP)); RET_ON_ERR(cudaMalloc(&dU0, szP)); RET_ON_ERR(cudaMalloc(&dU1, szP));
    RET_ON_ERR(cudaMalloc(&dRHS, szC));
    RET_ON_ERR(cudaMalloc(&dlam, (size_t)N * N * sizeof(R)));
    RET_ON_ERR(cudaMalloc(&dtmp, 65 * sizeof(R)));
    RET_ON_ERR(cudaMemcpy(dU, Uh, szP, cudaMemcpyHostToDevice));
    RET_ON_ERR(cudaMemset(dRHS, 0, szC));
    compute_rhs<<<GS_NBLK, BLOCK1D>>>(dU, dRHS, dlam, N, Np, h);
    RET_ON_ERR(cudaDeviceSynchronize());
    R lmax = gpu_max(dlam, dtmp, N * N), t = 0, dt = 0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    cudaEventRecord(e0);
    int step = 0, status = 0;
    while (step < max_steps && t < t_stop) {
        if (!(lmax > 0.)) { status = 1; break; }
        dt = cfl * h / lmax;
        if (t + dt > t_stop) dt = t_stop - t;
        if (dt < 1e-14) { status = 2; break; }
        RET_ON_ERR(cudaMemcpy(dU0, dU, szP, cudaMemcpyDeviceToDevice));
        rk_stage<<<GS_NBLK, BLOCK1D>>>(dU1, dU0, dU0, dRHS, 0., 1., 0., dt, N, Np);
        limit_positivity_blocks<<<GS_NBLK, BLOCK1D>>>(dU1, N, Np);
        apply_bc<<<GS_NBLK, BLOCK1D>>>(dU1, N, Np);
        RET_ON_ERR(cudaMemset(dRHS, 0, szC));
        compute_rhs<<<GS_NBLK, BLOCK1D>>>(dU1, dRHS, dlam, N, Np, h);
        rk_stage<<<GS_NBLK, BLOCK1D>>>(dU1, dU0, dU1, dRHS, 0.75, 0.25, 0., dt, N, Np);
        limit_positivity_blocks<<<GS_NBLK, BLOCK1D>>>(dU1, N, Np);
        apply_bc<<<GS_NBLK, BLOCK1D>>>(dU1, N, Np);
        RET_ON_ERR(cudaMemset(dRHS, 0, szC));
        compute_rhs<<<GS_NBLK, BLOCK1D>>>(dU1, dRHS, dlam, N, Np, h);
        rk_stage<<<GS_NBLK, BLOCK1D>>>(dU, dU0, dU1, dRHS, (R)(1. / 3.), (R)(2. / 3.), 0., dt, N, Np);
        limit_positivity_blocks<<<GS_NBLK, BLOCK1D>>>(dU, N, Np);
        apply_bc<<<GS_NBLK, BLOCK1D>>>(dU, N, Np);
        RET_ON_ERR(cudaMemset(dRHS, 0, szC));
        compute_rhs<<<GS_NBLK, BLOCK1D>>>(dU, dRHS, dlam, N, Np, h);
        RET_ON_ERR(cudaDeviceSynchronize());
        lmax = gpu_max(dlam, dtmp, N * N);
        t += dt;
        step++;
    }
    cudaEventRecord(e1);
    RET_ON_ERR(cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms_out) *ms_out = ms;
    RET_ON_ERR(cudaGetLastError());
    RET_ON_ERR(cudaMemcpy(Uh, dU, szP, cudaMemcpyDeviceToHost));
    if (info) { info[0] = t; info[1] = step; info[2] = lmax; info[3] = dt; }
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    cudaFree(dU); cudaFree(dU0); cudaFree(dU1); cudaFree(dRHS); cudaFree(dlam); cudaFree(dtmp);
    return status ? -status : 0;
}

}  /* extern "C" */
#endif
