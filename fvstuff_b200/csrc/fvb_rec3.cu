// fvb_rec3.cu -- the rec3 + HLLC + 2x2-block Zhang-Shu scheme of
// fv_rec3_2d.cu on the device (FP64, conserved cell averages, g = 2,
// periodic, N even).
//
// Per face: unlimited 3rd-order parabolic reconstruction of the conserved
// variables on both sides, each face state scaled toward its own cell's
// average until rho and p clear their floors (the pointwise Zhang-Shu
// scaling), conversion to floored primitives, HLLC.  Per cell: the residual,
// the SSP-RK3 combination, then the a-posteriori Zhang-Shu limiter on the
// non-overlapping 2x2 blocks of the new state (block corners by bilinear
// extrapolation, one common theta per block, block total conserved).
//
// One launch per stage does all of it for a tile of 32 x 32 cells: tiles
// start on even cells, so every 2x2 block lies in one tile, and after the
// face fluxes one thread takes one block -- the residuals and RK values of
// its four cells, the limiter, the stores (interior + periodic ghost
// images) -- with no barrier between; stage 3 max-reduces the wave speed of
// the limited state.
//
// The reference scatters each face flux into its two cells with atomicAdd;
// here every cell gathers its four face terms in the order a serial run of
// that scatter adds them (by source cell index), and this file is compiled
// without FMA contraction (-fmad=false), so each stage reproduces the
// reference's arithmetic operation for operation.
#include <algorithm>

#include "fvb_aux.h"
#include "fvb_device.cuh"

namespace fvb {
namespace {

constexpr double R3_GAM = 1.4, R3_PFLOOR = 1e-9, R3_RHOFLOOR = 1e-12;
constexpr int RTX = 32, RTY = 32, RNT = 256, RG = 2;
constexpr int RSW = RTX + 2 * RG, RSH = RTY + 2 * RG, RPL = RSW * RSH;
constexpr int RNC = RTX * RTY;

// c = sqrt(gamma p / rho)                       fv_rec3_2d.cu:68-69
__device__ __forceinline__ double r3_snd(double rho, double p) { return sqrt(R3_GAM * p / rho); }

// conserved point value -> floored primitives  fv_rec3_2d.cu:71-79
__device__ __forceinline__ void r3_w(const double U[4], double W[4])
{
    const double r = smax<double>(U[0], R3_RHOFLOOR);
    const double u = U[1] / r, v = U[2] / r;
    const double p = (R3_GAM - 1.0) * (U[3] - 0.5 * r * (u * u + v * v));
    W[0] = r; W[1] = u; W[2] = v; W[3] = smax<double>(p, R3_PFLOOR);
}

// pressure of a conserved state                fv_rec3_2d.cu:81-87
__device__ __forceinline__ double r3_p(const double U[4])
{
    const double r = smax<double>(U[0], R3_RHOFLOOR);
    const double u = U[1] / r, v = U[2] / r;
    return (R3_GAM - 1.0) * (U[3] - 0.5 * r * (u * u + v * v));
}

// HLLC with Davis bounds and each side's star state, in the face-normal
// frame (rho, un, ut, p); a y-face swaps (u, v) in and the momentum
// fluxes back, which for the normal (0, 1) equals the reference's rotation
// bit for bit                                  fv_rec3_2d.cu:90-123
__device__ void r3_hllc(const double L[4], const double R[4], double F[4])
{
    const double rL = L[0], uL = L[1], tL = L[2], pL = L[3];
    const double rR = R[0], uR = R[1], tR = R[2], pR = R[3];
    const double cL = r3_snd(rL, pL), cR = r3_snd(rR, pR);
    const double EL = pL / (R3_GAM - 1.) + 0.5 * rL * (uL * uL + tL * tL);
    const double ER = pR / (R3_GAM - 1.) + 0.5 * rR * (uR * uR + tR * tR);
    const double SL = smin<double>(uL - cL, uR - cR), SR = smax<double>(uL + cL, uR + cR);
    const double FL[4] = {rL * uL, rL * uL * uL + pL, rL * uL * tL, (EL + pL) * uL};
    const double FR[4] = {rR * uR, rR * uR * uR + pR, rR * uR * tR, (ER + pR) * uR};
    if (SL >= 0.) { for (int q = 0; q < 4; q++) F[q] = FL[q]; return; }
    if (SR <= 0.) { for (int q = 0; q < 4; q++) F[q] = FR[q]; return; }
    const double dL = rL * (SL - uL), dR = rR * (SR - uR);
    const double Ss = (pR - pL + dL * uL - dR * uR) / (dL - dR);
    const bool left = Ss >= 0.;
    const double rK = left ? rL : rR, uK = left ? uL : uR, tK = left ? tL : tR, pK = left ? pL : pR;
    const double EK = left ? EL : ER, SK = left ? SL : SR;
    const double f = rK * (SK - uK) / (SK - Ss);
    const double Us[4] = {f, f * Ss, f * tK, f * (EK / rK + (Ss - uK) * (Ss + pK / (rK * (SK - uK))))};
    const double U[4] = {rK, rK * uK, rK * tK, EK};
    for (int q = 0; q < 4; q++) F[q] = (left ? FL[q] : FR[q]) + SK * (Us[q] - U[q]);
}

// Zhang-Shu scaling of a face state toward its cell average (linear for
// rho, 25-step bisection for p), then its floored primitives: the density,
// velocity and pressure that the pressure test forms are the primitives'
// own unless the bisection moved the state, so they are reused (the same
// operations on the same values as scaling, then converting)
//                                               fv_rec3_2d.cu:125-145, :71-79
__device__ __forceinline__ void r3_scale_w(const double Ub[4], double U[4], double W[4])
{
    if (U[0] < R3_RHOFLOOR) {
        const double d = Ub[0] - U[0];
        const double th = (d > 0.) ? (Ub[0] - R3_RHOFLOOR) / d : 0.;
        for (int q = 0; q < 4; q++) U[q] = Ub[q] + th * (U[q] - Ub[q]);
    }
    double r = smax<double>(U[0], R3_RHOFLOOR);
    double u = U[1] / r, v = U[2] / r;
    double p = (R3_GAM - 1.0) * (U[3] - 0.5 * r * (u * u + v * v));
    if (p < R3_PFLOOR) {
        double lo = 0., hi = 1.;
        for (int it = 0; it < 25; it++) {
            const double mid = 0.5 * (lo + hi);
            double V[4];
            for (int q = 0; q < 4; q++) V[q] = Ub[q] + mid * (U[q] - Ub[q]);
            if (V[0] >= R3_RHOFLOOR && r3_p(V) >= R3_PFLOOR) lo = mid;
            else hi = mid;
        }
        for (int q = 0; q < 4; q++) U[q] = Ub[q] + lo * (U[q] - Ub[q]);
        r = smax<double>(U[0], R3_RHOFLOOR);
        u = U[1] / r;
        v = U[2] / r;
        p = (R3_GAM - 1.0) * (U[3] - 0.5 * r * (u * u + v * v));
    }
    W[0] = r; W[1] = u; W[2] = v; W[3] = smax<double>(p, R3_PFLOOR);
}

// 2x2-block limiter on U[c][q] (cells c = 0..3: (i0,j0), (i0+1,j0),
// (i0,j0+1), (i0+1,j0+1)); true if the block changed; *brutal counts a
// block whose mean itself needed the floor fix  fv_rec3_2d.cu:252-337
__device__ bool r3_limit_block(double U[4][4], int *brutal)
{
    double Ub[4] = {0., 0., 0., 0.};
    for (int c = 0; c < 4; c++)
        for (int q = 0; q < 4; q++) Ub[q] += 0.25 * U[c][q];
    const double pb = r3_p(Ub);
    if (Ub[0] < R3_RHOFLOOR || pb < R3_PFLOOR) {
        ++*brutal;
        const double rb = smax<double>(Ub[0], 10. * R3_RHOFLOOR);
        const double Efix = (10. * R3_PFLOOR) / (R3_GAM - 1.) + 0.5 * (Ub[1] * Ub[1] + Ub[2] * Ub[2]) / rb;
        Ub[0] = rb;
        Ub[3] = smax<double>(Ub[3], Efix);
    }
    double C[4][4];
    for (int q = 0; q < 4; q++) {
        C[0][q] = (9. * U[0][q] - 3. * U[1][q] - 3. * U[2][q] + U[3][q]) * 0.25;
        C[1][q] = (9. * U[1][q] - 3. * U[0][q] - 3. * U[3][q] + U[2][q]) * 0.25;
        C[2][q] = (9. * U[2][q] - 3. * U[3][q] - 3. * U[0][q] + U[1][q]) * 0.25;
        C[3][q] = (9. * U[3][q] - 3. * U[2][q] - 3. * U[1][q] + U[0][q]) * 0.25;
    }
    double th = 1.;
    for (int c = 0; c < 4; c++)
        if (C[c][0] < R3_RHOFLOOR) {
            const double d = Ub[0] - C[c][0];
            if (d > 0.) th = smin<double>((Ub[0] - R3_RHOFLOOR) / d, th);
        }
    if (th < 1.)
        for (int c = 0; c < 4; c++)
            for (int q = 0; q < 4; q++) {
                U[c][q] = Ub[q] + th * (U[c][q] - Ub[q]);
                C[c][q] = Ub[q] + th * (C[c][q] - Ub[q]);
            }
    bool bad = false;
    for (int c = 0; c < 4; c++)
        if (C[c][0] < R3_RHOFLOOR || r3_p(C[c]) < R3_PFLOOR) bad = true;
    if (bad) {
        double lo = 0., hi = 1.;
        for (int it = 0; it < 30; it++) {
            const double mid = 0.5 * (lo + hi);
            bool ok = true;
            for (int c = 0; c < 4 && ok; c++) {
                double V[4];
                for (int q = 0; q < 4; q++) V[q] = Ub[q] + mid * (C[c][q] - Ub[q]);
                if (V[0] < R3_RHOFLOOR || r3_p(V) < R3_PFLOOR) ok = false;
            }
            if (ok) lo = mid;
            else hi = mid;
        }
        for (int c = 0; c < 4; c++)
            for (int q = 0; q < 4; q++) U[c][q] = Ub[q] + lo * (U[c][q] - Ub[q]);
    }
    return th < 1. || bad;
}

__device__ __forceinline__ long long r3_at(const GridDev &gd, int j, int i)
{
    return (long long)(j + RG) * gd.pitch + (i + RG) + gd.xoff;
}

// one SSP-RK3 stage                             fv_rec3_2d.cu:166-353
__global__ void __launch_bounds__(RNT, 2) rec3_stage_kernel(const GridDev gd, int stage, int ntiles)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *Q = reinterpret_cast<double *>(smem_raw);  // [4][RSH][RSW] stage input
    double *FX = Q + 4 * RPL;                          // [4][RTY][RTX+1]
    double *FY = FX + 4 * RTY * (RTX + 1);             // [4][RTY+1][RTX]
    __shared__ TileCtl s_ctl;
    __shared__ double s_red[RNT / 32];
    const int tid = threadIdx.x, n = gd.n, np = n + 2 * RG;
    const double *in = (const double *)(stage == 2 ? gd.k1 : stage == 3 ? gd.k2 : gd.st[0]);
    const double *u0 = (const double *)gd.st[0];
    double *out = (double *)(stage == 1 ? gd.k1 : stage == 2 ? gd.k2 : gd.st[0]);
    const double inv_h = 1. / gd.h;
    const double ca = stage == 1 ? 0. : stage == 2 ? 0.75 : 1. / 3.;
    const double cb = stage == 1 ? 1. : stage == 2 ? 0.25 : 2. / 3.;
    int brutal = 0;
    double lacc = 0.0;

    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int tx0 = (t % gd.tiles_x) * RTX, ty0 = (t / gd.tiles_x) * RTY;
        if (tid == 0) s_ctl = tile_control<P64>(gd.ctrl, stage, t == 0);
        __syncthreads();
        const TileCtl ctl = s_ctl;
        if (!ctl.run) {
            __syncthreads();
            continue;
        }
        // ---- halo box of the stage input (an admissible dummy outside) ----
        for (int k = tid; k < RPL; k += RNT) {
            const int r = k / RSW, c = k - r * RSW, jp = ty0 + r, ip = tx0 + c;
            const bool inb = jp < np && ip < np;
            const long long e = (long long)jp * gd.pitch + ip + gd.xoff;
            for (int q = 0; q < 4; ++q) Q[q * RPL + k] = inb ? in[e + q * gd.plane] : (q == 0 ? 1. : q == 3 ? 2.5 : 0.);
        }
        __syncthreads();
        // ---- faces: x-face (r, c) lies between cells c-1 and c ------------
        for (int f = tid; f < (RTX + 1) * RTY + RTX * (RTY + 1); f += RNT) {
            const bool xf = f < (RTX + 1) * RTY;
            int r, c, st;
            if (xf) { r = f / (RTX + 1); c = f - r * (RTX + 1); st = 1; }
            else { const int f2 = f - (RTX + 1) * RTY; r = f2 / RTX; c = f2 - r * RTX; st = RSW; }
            const int b = (r + RG) * RSW + (c + RG), a = b - st;
            double UL[4], UR[4], UbL[4], UbR[4];
            for (int q = 0; q < 4; ++q) {
                const double *v = Q + q * RPL;
                const double um = v[a - st], uc = v[a], up = v[b], u2 = v[b + st];
                UL[q] = (-um + 5. * uc + 2. * up) * (1. / 6.);
                UR[q] = (2. * uc + 5. * up - u2) * (1. / 6.);
                UbL[q] = uc;
                UbR[q] = up;
            }
            double WL[4], WR[4], L[4], Rr[4], Fn[4];
            r3_scale_w(UbL, UL, WL);
            r3_scale_w(UbR, UR, WR);
            const int QN = xf ? 1 : 2, QT = xf ? 2 : 1;
            L[0] = WL[0]; L[1] = WL[QN]; L[2] = WL[QT]; L[3] = WL[3];
            Rr[0] = WR[0]; Rr[1] = WR[QN]; Rr[2] = WR[QT]; Rr[3] = WR[3];
            r3_hllc(L, Rr, Fn);
            double *o = xf ? FX + r * (RTX + 1) + c : FY + r * RTX + c;
            const int os = xf ? RTY * (RTX + 1) : (RTY + 1) * RTX;
            o[0] = Fn[0]; o[QN * os] = Fn[1]; o[QT * os] = Fn[2]; o[3 * os] = Fn[3];
        }
        __syncthreads();
        // ---- per 2x2 block, one thread: residual of its four cells in the
        //      serial scatter's order, RK combination, the block limiter,
        //      stores with the periodic ghost images, stage-3 wave speed -----
        for (int kb = tid; kb < RNC / 4; kb += RNT) {
            const int jb = kb / (RTX / 2), ib = kb - jb * (RTX / 2);
            const int c0 = 2 * ib, r0 = 2 * jb;
            if (tx0 + c0 >= n || ty0 + r0 >= n) continue;  // n even: the block is whole
            double U[4][4];
            for (int cc = 0; cc < 4; cc++) {
                const int r = r0 + (cc >> 1), c = c0 + (cc & 1), i = tx0 + c, j = ty0 + r;
                const long long e = r3_at(gd, j, i);
                for (int q = 0; q < 4; ++q) {
                    const double *fx = FX + q * RTY * (RTX + 1) + r * (RTX + 1) + c;
                    const double *fy = FY + q * (RTY + 1) * RTX + r * RTX + c;
                    const double tl = fx[0] * inv_h, tr = -fx[1] * inv_h;      // left face in, right face out
                    const double tb = fy[0] * inv_h, tt = -fy[RTX] * inv_h;    // bottom in, top out
                    double L;
                    if (i > 0 && j > 0) L = ((tb + tl) + tr) + tt;
                    else if (i == 0 && j > 0) L = ((tb + tr) + tt) + tl;
                    else if (i > 0) L = ((tl + tr) + tt) + tb;
                    else L = ((tr + tt) + tl) + tb;
                    const double qa = u0[e + q * gd.plane];
                    const double qb = Q[q * RPL + (r + RG) * RSW + (c + RG)];
                    U[cc][q] = ca * qa + cb * (qb + ctl.dt * L);
                }
            }
            r3_limit_block(U, &brutal);
            for (int cc = 0; cc < 4; cc++) {
                const int i = tx0 + c0 + (cc & 1), j = ty0 + r0 + (cc >> 1);
                put_cell<double>(gd, out, j, i, U[cc]);
                if (stage == 3) {
                    double W[4];
                    r3_w(U[cc], W);
                    lacc = smax<double>(fabs(W[1]) + fabs(W[2]) + r3_snd(W[0], W[3]), lacc);
                }
            }
        }
        if (stage == 3 && tid == 0 && t == 0) leader_finish<P64>(gd.ctrl);
        __syncthreads();
    }
    if (brutal) atomicAdd(&gd.ctrl->aux, (unsigned long long)brutal);
    if (stage == 3) {
        for (int o = 16; o > 0; o >>= 1) lacc = fmax(lacc, __shfl_xor_sync(0xffffffffu, lacc, o));
        if ((tid & 31) == 0) s_red[tid >> 5] = lacc;
        __syncthreads();
        if (tid == 0) {
            double m = 0.0;
            for (int w = 0; w < RNT / 32; ++w) m = fmax(m, s_red[w]);
            if (m > 0.0) atomicMax(&gd.ctrl->lam_acc, (unsigned long long)__double_as_longlong(m));
        }
    }
}

// limiter pass over a whole state (after an initial state is set), one
// thread per 2x2 block                          fv_rec3_2d.cu:542
__global__ void rec3_limit_kernel(const GridDev gd, double *buf)
{
    const int nb = gd.n / 2;
    int brutal = 0;
    for (long long kb = blockIdx.x * (long long)blockDim.x + threadIdx.x; kb < (long long)nb * nb;
         kb += (long long)blockDim.x * gridDim.x) {
        const int jb = (int)(kb / nb), ib = (int)(kb - (long long)jb * nb);
        double U[4][4];
        for (int cc = 0; cc < 4; cc++) {
            const long long e = r3_at(gd, 2 * jb + (cc >> 1), 2 * ib + (cc & 1));
            for (int q = 0; q < 4; q++) U[cc][q] = buf[e + q * gd.plane];
        }
        if (r3_limit_block(U, &brutal))
            for (int cc = 0; cc < 4; cc++) {
                const long long e = r3_at(gd, 2 * jb + (cc >> 1), 2 * ib + (cc & 1));
                for (int q = 0; q < 4; q++) buf[e + q * gd.plane] = U[cc][q];
            }
    }
    if (brutal) atomicAdd(&gd.ctrl->aux, (unsigned long long)brutal);
}

// |u| + |v| + c of the floored primitives, max into ctrl->lam_acc
__global__ void rec3_lam_kernel(const GridDev gd, const double *buf)
{
    __shared__ double sh[32];
    const long long n2 = (long long)gd.n * gd.n;
    double m = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n2;
         k += (long long)blockDim.x * gridDim.x) {
        const long long e = r3_at(gd, (int)(k / gd.n), (int)(k % gd.n));
        double U[4], W[4];
        for (int q = 0; q < 4; q++) U[q] = buf[e + q * gd.plane];
        r3_w(U, W);
        m = fmax(m, fabs(W[1]) + fabs(W[2]) + r3_snd(W[0], W[3]));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b = fmax(b, sh[w]);
        atomicMax(&gd.ctrl->lam_acc, (unsigned long long)__double_as_longlong(b));
    }
}

// initial cell averages of fv_rec3's cases: 0 circular Sod (sharp,
// midpoint), 1 the paper's isentropic vortex on [0,10]^2, 2 the Gresho
// low-Mach vortex; 4x4 Gauss averages for the smooth ones
//                                               fv_rec3_2d.cu:356-416
__device__ void r3_pv(double x, double y, double *ro, double *uo, double *vo, double *po)
{
    const double gg = R3_GAM, eps = 5., pi = 3.14159265358979323846;
    const double dx = x - 5., dy = y - 5., r2 = dx * dx + dy * dy;
    const double f = eps / (2. * pi) * exp(0.5 * (1. - r2));
    const double dT = -(gg - 1.) * eps * eps / (8. * gg * pi * pi) * exp(1. - r2);
    double T = 1. + dT;
    if (T < 1e-6) T = 1e-6;
    *ro = pow(T, 1. / (gg - 1.));
    *po = pow(T, gg / (gg - 1.));
    *uo = -f * dy;
    *vo = f * dx;
}
__device__ void r3_lmv(double x, double y, double p0, double *ro, double *uo, double *vo, double *po)
{
    const double dx = x - 0.5, dy = y - 0.5, r = sqrt(dx * dx + dy * dy);
    const double vp = r < 0.2 ? 5. * r : r < 0.4 ? 2. - 5. * r : 0.;
    const double ir = (r > 1e-30) ? 1. / r : 0.;
    *ro = 1.; *uo = -vp * dy * ir; *vo = vp * dx * ir;
    *po = r < 0.2 ? p0 + 12.5 * r * r : r < 0.4 ? p0 + 4. * log(5. * r) + 4. - 20. * r + 12.5 * r * r
                                                : p0 + 4. * log(2.) - 2.;
}

__global__ void rec3_ic_kernel(const GridDev gd, double *buf, int icase, double p0)
{
    const double gx[4] = {-0.861136311594053, -0.339981043584856, 0.339981043584856, 0.861136311594053};
    const double gw[4] = {0.347854845137454, 0.652145154862546, 0.652145154862546, 0.347854845137454};
    const int n = gd.n;
    const double h = gd.h;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < (long long)n * n;
         k += (long long)blockDim.x * gridDim.x) {
        const int j = (int)(k / n), i = (int)(k % n);
        const double xc = (i + 0.5) * h, yc = (j + 0.5) * h;
        double Qc[4] = {0., 0., 0., 0.};
        if (icase == 0) {
            const double r = sqrt((xc - 0.5) * (xc - 0.5) + (yc - 0.5) * (yc - 0.5));
            Qc[0] = r < 0.25 ? 10.0 : 0.125;
            Qc[3] = (r < 0.25 ? 10.0 : 0.1) / (R3_GAM - 1.);
        } else {
            for (int a = 0; a < 4; a++)
                for (int b = 0; b < 4; b++) {
                    const double x = xc + 0.5 * h * gx[a], y = yc + 0.5 * h * gx[b];
                    double r, u, v, p;
                    if (icase == 1) r3_pv(x, y, &r, &u, &v, &p);
                    else r3_lmv(x, y, p0, &r, &u, &v, &p);
                    const double w = 0.25 * gw[a] * gw[b];
                    Qc[0] += w * r; Qc[1] += w * r * u; Qc[2] += w * r * v;
                    Qc[3] += w * (p / (R3_GAM - 1.) + 0.5 * r * (u * u + v * v));
                }
        }
        const long long e = r3_at(gd, j, i);
        for (int q = 0; q < 4; q++) buf[e + q * gd.plane] = Qc[q];
    }
}

size_t rec3_smem()
{
    return sizeof(double) * (4 * RPL + 4 * RTY * (RTX + 1) + 4 * (RTY + 1) * RTX);
}

int sm_count()
{
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

}  // namespace

void rec3_tiles(int n, int &tiles_x, int &tiles)
{
    tiles_x = (n + RTX - 1) / RTX;
    tiles = tiles_x * ((n + RTY - 1) / RTY);
}

cudaError_t rec3_launch_stage(const GridDev &gd, int stage, int tiles, cudaStream_t s)
{
    LaunchFacts f{};
    cudaError_t e = launch_facts((const void *)rec3_stage_kernel, RNT, rec3_smem(), f);
    if (e != cudaSuccess) return e;
    const int cap = f.ctas_per_sm * f.sms;
    rec3_stage_kernel<<<tiles < cap ? tiles : cap, RNT, rec3_smem(), s>>>(gd, stage, tiles);
    return cudaGetLastError();
}

cudaError_t rec3_limit_into(const GridDev &gd, void *buf, cudaStream_t s)
{
    const long long nb = (long long)(gd.n / 2) * (gd.n / 2);
    const int blocks = (int)std::min<long long>((nb + 255) / 256, 4LL * sm_count());
    rec3_limit_kernel<<<blocks > 0 ? blocks : 1, 256, 0, s>>>(gd, (double *)buf);
    return cudaGetLastError();
}

cudaError_t rec3_lam_into(const GridDev &gd, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(&gd.ctrl->lam_acc, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    const long long n2 = (long long)gd.n * gd.n;
    const int blocks = (int)std::min<long long>((n2 + 255) / 256, 4LL * sm_count());
    rec3_lam_kernel<<<blocks, 256, 0, s>>>(gd, (const double *)gd.st[0]);
    return cudaGetLastError();
}

cudaError_t rec3_init_case(const GridDev &gd, int icase, double p0, cudaStream_t s)
{
    const long long n2 = (long long)gd.n * gd.n;
    const int blocks = (int)std::min<long long>((n2 + 255) / 256, 4LL * sm_count());
    rec3_ic_kernel<<<blocks, 256, 0, s>>>(gd, (double *)gd.st[0], icase, p0);
    return cudaGetLastError();
}

}  // namespace fvb
