// fvb_d2av.cu -- the scheme kept in fv_up7_ducros_2d.cu.bak (the earlier
// form of fv_up7) on the device: UP-order (3, 5, 7, 9) reconstruction of the
// conserved variables, HLLC on the reconstructed states, and a D2
// artificial viscosity
//   D2 = (C2/h) S_D (sum of lam_face dU) + (Cg/h) (1 - S_D) (the same sum)
// whose Ducros weight S_D = div^2 / (div^2 + sc c^2 / h^2) comes from the
// 6th-order divergence of the velocity (compressions only).  SSP-RK3 on
// conserved variables, no floors; FP64.
//
// One launch per stage does all of it for a tile of 32 x 8 cells: the halo
// box of the stage input (g = max((order+1)/2, 3) layers, the sensor's reach)
// goes to shared memory together with each box cell's sensor velocities,
// |u|+c, |v|+c and c; every face flux is computed once; each cell then
// forms its residual, sensor and viscosity, combines the RK stage and stores
// itself with its ghost images (put_cell).  Stage 3 max-reduces |u|+|v|+c of
// the new state for the next step's dt.
//
// Every expression keeps the reference's association order and this file
// is compiled without FMA contraction (-fmad=false), so a stage reproduces
// the reference kernels' arithmetic operation for operation.
#include <algorithm>

#include "fvb_aux.h"
#include "fvb_device.cuh"

namespace fvb {
namespace {

constexpr int DTX = 32, DTY = 8, DNT = 256;

// conserved -> p, c, u, v; no density floor, c^2 floored at 1e-14
//                                          fv_up7_ducros_2d.cu.bak:65-74
__device__ __forceinline__ void d2_prim(double gam, double rho, double mx, double my, double E, double &p,
                                        double &c, double &u, double &v)
{
    u = mx / rho;
    v = my / rho;
    p = (gam - 1.0) * (E - 0.5 * (mx * u + my * v));
    const double cs2 = gam * p / rho;
    c = sqrt(cs2 > 1e-14 ? cs2 : 1e-14);
}

// HLLC of conserved face states in the face-normal frame (rho, m_n, m_t, E);
// a y-face passes (rho v, rho u) as (m_n, m_t), which leaves every
// operation's operands as the reference's y-solver has them
//                                          fv_up7_ducros_2d.cu.bak:202-282
__device__ void d2_hllc(double gam, const double UL[4], const double UR[4], double F[4])
{
    double pL, cL, uL, vL, pR, cR, uR, vR;
    d2_prim(gam, UL[0], UL[1], UL[2], UL[3], pL, cL, uL, vL);
    d2_prim(gam, UR[0], UR[1], UR[2], UR[3], pR, cR, uR, vR);
    const double SL = smin<double>(uL - cL, uR - cR);
    const double SR = smax<double>(uL + cL, uR + cR);
    if (SL >= 0.0) {
        F[0] = UL[1]; F[1] = UL[1] * uL + pL; F[2] = UL[1] * vL; F[3] = (UL[3] + pL) * uL;
        return;
    }
    if (SR <= 0.0) {
        F[0] = UR[1]; F[1] = UR[1] * uR + pR; F[2] = UR[1] * vR; F[3] = (UR[3] + pR) * uR;
        return;
    }
    const double dL = UL[0] * (SL - uL), dR = UR[0] * (SR - uR);
    const double Ss = (pR - pL + dL * uL - dR * uR) / (dL - dR);
    const bool left = Ss >= 0.0;
    const double K0 = left ? UL[0] : UR[0], K1 = left ? UL[1] : UR[1];
    const double K2 = left ? UL[2] : UR[2], K3 = left ? UL[3] : UR[3];
    const double pK = left ? pL : pR, uK = left ? uL : uR, vK = left ? vL : vR, SK = left ? SL : SR;
    const double f = K0 * (SK - uK) / (SK - Ss);
    const double s3 = f * (K3 / K0 + (Ss - uK) * (Ss + pK / (K0 * (SK - uK))));
    F[0] = K1 + SK * (f - K0);
    F[1] = (K1 * uK + pK) + SK * (f * Ss - K1);
    F[2] = K1 * vK + SK * (f * vK - K2);
    F[3] = (K3 + pK) * uK + SK * (s3 - K3);
}

// upwind-biased face values from the stencil s[0 .. order] along the face
// normal (the face lies between s[hw-1] and s[hw])
//                                          fv_up7_ducros_2d.cu.bak:105-153
template <int ORDER>
__device__ __forceinline__ void d2_recon(const double *s, double &vL, double &vR)
{
    if constexpr (ORDER == 3) {
        vL = (-s[0] + 5.0 * s[1] + 2.0 * s[2]) / 6.0;
        vR = (2.0 * s[1] + 5.0 * s[2] - s[3]) / 6.0;
    } else if constexpr (ORDER == 5) {
        vL = (2.0 * s[0] - 13.0 * s[1] + 47.0 * s[2] + 27.0 * s[3] - 3.0 * s[4]) / 60.0;
        vR = (-3.0 * s[1] + 27.0 * s[2] + 47.0 * s[3] - 13.0 * s[4] + 2.0 * s[5]) / 60.0;
    } else if constexpr (ORDER == 9) {
        // the published weights as they stand (the left-biased set sums to
        // 4217/2520)                            fv_up7_ducros_2d.cu.bak:132-142
        vL = (3.0 * s[0] - 25.0 * s[1] + 101.0 * s[2] - 319.0 * s[3] + 2765.0 * s[4] + 2139.0 * s[5] -
              533.0 * s[6] + 97.0 * s[7] - 11.0 * s[8]) /
             2520.0;
        vR = (-11.0 * s[1] + 97.0 * s[2] - 533.0 * s[3] + 2139.0 * s[4] + 2765.0 * s[5] - 319.0 * s[6] +
              101.0 * s[7] - 25.0 * s[8] + 3.0 * s[9]) /
             2520.0;
    } else {
        vL = (-3.0 * s[0] + 25.0 * s[1] - 101.0 * s[2] + 319.0 * s[3] + 214.0 * s[4] - 38.0 * s[5] + 4.0 * s[6]) /
             420.0;
        vR = (4.0 * s[1] - 38.0 * s[2] + 214.0 * s[3] + 319.0 * s[4] - 101.0 * s[5] + 25.0 * s[6] - 3.0 * s[7]) /
             420.0;
    }
}

template <int ORDER>
struct D2Shape {
    static constexpr int HW = (ORDER + 1) / 2;         // reconstruction half width
    static constexpr int HB = HW > 3 ? HW : 3;         // halo of the box (= the grid's ghost width)
    static constexpr int BW = DTX + 2 * HB, BH = DTY + 2 * HB, PL = BW * BH;
    static constexpr int NFX = (DTX + 1) * DTY, NFY = DTX * (DTY + 1);
    // Q[4][PL] | SU, SV, LX, LY, CS [PL each] | FX[4][NFX] | FY[4][NFY]
    static constexpr size_t SMEM = sizeof(double) * (9 * PL + 4 * NFX + 4 * NFY);
    // resident CTAs an SM is compiled for: four (56 KB each, <= 64
    // registers) with the 3-cell halo, three (64 KB, 72 KB) with UP7's 4
    // and UP9's 5
    static constexpr int MINB = HB == 3 ? 4 : 3;
};

// one SSP-RK3 stage                        fv_up7_ducros_2d.cu.bak:287-446
template <int ORDER>
__global__ void __launch_bounds__(DNT, D2Shape<ORDER>::MINB)
    d2av_stage_kernel(const GridDev gd, int stage, int ntiles, D2Params av)
{
    using S = D2Shape<ORDER>;
    constexpr int HW = S::HW, HB = S::HB, BW = S::BW, PL = S::PL;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *Q = reinterpret_cast<double *>(smem_raw);  // [4][BH][BW] stage input
    double *SU = Q + 4 * PL;                           // rho u / max(rho, 1e-14)
    double *SV = SU + PL;                              // rho v / max(rho, 1e-14)
    double *LX = SV + PL;                              // |u| + c
    double *LY = LX + PL;                              // |v| + c
    double *CS = LY + PL;                              // c
    double *FX = CS + PL;                              // [4][DTY][DTX+1]
    double *FY = FX + 4 * S::NFX;                      // [4][DTY+1][DTX]
    __shared__ TileCtl s_ctl;
    __shared__ double s_red[DNT / 32];
    const int tid = threadIdx.x, n = gd.n, np = n + 2 * HB;
    const double gam = gd.gam, h = gd.h;
    const double *in = (const double *)(stage == 2 ? gd.k1 : stage == 3 ? gd.k2 : gd.st[0]);
    const double *u0 = (const double *)gd.st[0];
    double *out = (double *)(stage == 1 ? gd.k1 : stage == 2 ? gd.k2 : gd.st[0]);
    double lacc = 0.0;

    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int tx0 = (t % gd.tiles_x) * DTX, ty0 = (t / gd.tiles_x) * DTY;
        if (tid == 0) s_ctl = tile_control<P64>(gd.ctrl, stage, t == 0);
        __syncthreads();
        const TileCtl ctl = s_ctl;
        if (!ctl.run) {
            __syncthreads();
            continue;
        }
        // ---- halo box of the stage input and its per-cell quantities ------
        for (int k = tid; k < PL; k += DNT) {
            const int r = k / BW, c = k - r * BW, jp = ty0 + r, ip = tx0 + c;
            double U[4] = {1.0, 0.0, 0.0, 2.5};  // admissible filler beyond the padded grid
            if (jp < np && ip < np) {
                const long long e = (long long)jp * gd.pitch + ip + gd.xoff;
#pragma unroll
                for (int q = 0; q < 4; ++q) U[q] = in[e + q * gd.plane];
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) Q[q * PL + k] = U[q];
            const double rf = U[0] > 1e-14 ? U[0] : 1e-14;
            SU[k] = U[1] / rf;
            SV[k] = U[2] / rf;
            double p, cc, u, v;
            d2_prim(gam, U[0], U[1], U[2], U[3], p, cc, u, v);
            LX[k] = fabs(u) + cc;
            LY[k] = fabs(v) + cc;
            CS[k] = cc;
        }
        __syncthreads();
        // ---- faces: x-face (r, c) between tile cells c-1 and c, y-face
        //      (r, c) between rows r-1 and r; b = the right / top cell -----
        for (int f = tid; f < S::NFX + S::NFY; f += DNT) {
            const bool xf = f < S::NFX;
            int r, c, st;
            if (xf) { r = f / (DTX + 1); c = f - r * (DTX + 1); st = 1; }
            else { const int f2 = f - S::NFX; r = f2 / DTX; c = f2 - r * DTX; st = BW; }
            const int b = (r + HB) * BW + (c + HB);
            double L[4], R[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                double s[2 * HW];
#pragma unroll
                for (int d = 0; d < 2 * HW; ++d) s[d] = Q[q * PL + b + (d - HW) * st];
                d2_recon<ORDER>(s, L[q], R[q]);
            }
            const int qn = xf ? 1 : 2, qt = xf ? 2 : 1;
            const double UL[4] = {L[0], xf ? L[1] : L[2], xf ? L[2] : L[1], L[3]};
            const double UR[4] = {R[0], xf ? R[1] : R[2], xf ? R[2] : R[1], R[3]};
            double Fn[4];
            d2_hllc(gam, UL, UR, Fn);
            double *o = xf ? FX + r * (DTX + 1) + c : FY + r * DTX + c;
            const int os = xf ? S::NFX : S::NFY;
            o[0] = Fn[0];
            o[qn * os] = Fn[1];
            o[qt * os] = Fn[2];
            o[3 * os] = Fn[3];
        }
        __syncthreads();
        // ---- cells: residual, sensor, viscosity, RK combination, stores ---
        for (int k = tid; k < DTX * DTY; k += DNT) {
            const int r = k / DTX, c = k - r * DTX, i = tx0 + c, j = ty0 + r;
            if (i >= n || j >= n) continue;
            const int b = (r + HB) * BW + (c + HB);
            // Ducros weight                fv_up7_ducros_2d.cu.bak:344-357
            const double wc[6] = {-1., 9., -45., 45., -9., 1.};
            const int wo[6] = {-3, -2, -1, 1, 2, 3};
            double du_dx = 0., dv_dy = 0.;
#pragma unroll
            for (int m = 0; m < 6; ++m) {
                du_dx += wc[m] * SU[b + wo[m]];
                dv_dy += wc[m] * SV[b + wo[m] * BW];
            }
            du_dx /= 60. * h;
            dv_dy /= 60. * h;
            double div_u = du_dx + dv_dy;
            if (div_u > 0.) div_u = 0.;
            const double c0 = CS[b];
            const double sos2 = (av.sc / (h * h)) * c0 * c0;
            const double S_D = (div_u * div_u) / (div_u * div_u + sos2 + 1e-40);
            // face-averaged directional wave speeds   :359-367
            const double lamx_c = LX[b], lamy_c = LY[b];
            const double lhxp = 0.5 * (lamx_c + LX[b + 1]);
            const double lhxm = 0.5 * (lamx_c + LX[b - 1]);
            const double lhyp = 0.5 * (lamy_c + LY[b + BW]);
            const double lhym = 0.5 * (lamy_c + LY[b - BW]);
            const long long e = (long long)(j + HB) * gd.pitch + (i + HB) + gd.xoff;
            double v[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double *Qq = Q + q * PL;
                const double Uc = Qq[b];
                const double dxp = Qq[b + 1] - Uc, dxm = Uc - Qq[b - 1];
                const double dyp = Qq[b + BW] - Uc, dym = Uc - Qq[b - BW];
                const double d2_duc = (av.c2 / h) * (lhxp * S_D * dxp - lhxm * S_D * dxm + lhyp * S_D * dyp -
                                                     lhym * S_D * dym);
                const double d2_glb = (av.cg / h) * (lhxp * (1. - S_D) * dxp - lhxm * (1. - S_D) * dxm +
                                                     lhyp * (1. - S_D) * dyp - lhym * (1. - S_D) * dym);
                const double D2 = d2_duc + d2_glb;
                const double *fx = FX + q * S::NFX + r * (DTX + 1) + c;
                const double *fy = FY + q * S::NFY + r * DTX + c;
                const double L = -(fx[1] - fx[0]) / h - (fy[DTX] - fy[0]) / h + D2;  // :386
                const double ua = u0[e + q * gd.plane];
                if (stage == 1) v[q] = ua + ctl.dt * L;                                   // :433-435
                else if (stage == 2) v[q] = 0.75 * ua + 0.25 * (Uc + ctl.dt * L);         // :437-440
                else v[q] = (1. / 3.) * ua + (2. / 3.) * (Uc + ctl.dt * L);               // :442-445
            }
            put_cell<double>(gd, out, j, i, v);
            if (stage == 3) {
                double p, cc, u, w;
                d2_prim(gam, v[0], v[1], v[2], v[3], p, cc, u, w);
                lacc = smax<double>(fabs(u) + fabs(w) + cc, lacc);  // lam_c, :362
            }
        }
        if (stage == 3 && tid == 0 && t == 0) leader_finish<P64>(gd.ctrl);
        __syncthreads();
    }
    if (stage == 3) {
        for (int o = 16; o > 0; o >>= 1) lacc = fmax(lacc, __shfl_xor_sync(0xffffffffu, lacc, o));
        if ((tid & 31) == 0) s_red[tid >> 5] = lacc;
        __syncthreads();
        if (tid == 0) {
            double m = 0.0;
            for (int w = 0; w < DNT / 32; ++w) m = fmax(m, s_red[w]);
            if (m > 0.0) atomicMax(&gd.ctrl->lam_acc, (unsigned long long)__double_as_longlong(m));
        }
    }
}

__device__ __forceinline__ long long d2_at(const GridDev &gd, int j, int i)
{
    return (long long)(j + gd.g) * gd.pitch + (i + gd.g) + gd.xoff;
}

// |u| + |v| + c of a state, max into ctrl->lam_acc      :77-83, :593-612
__global__ void d2av_lam_kernel(const GridDev gd, const double *buf)
{
    __shared__ double sh[32];
    const long long n2 = (long long)gd.n * gd.n;
    double m = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n2;
         k += (long long)blockDim.x * gridDim.x) {
        const long long e = d2_at(gd, (int)(k / gd.n), (int)(k % gd.n));
        double p, c, u, v;
        d2_prim(gd.gam, buf[e], buf[e + gd.plane], buf[e + 2 * gd.plane], buf[e + 3 * gd.plane], p, c, u, v);
        m = fmax(m, fabs(u) + fabs(v) + c);
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b = fmax(b, sh[w]);
        if (b > 0.0) atomicMax(&gd.ctrl->lam_acc, (unsigned long long)__double_as_longlong(b));
    }
}

// Ducros weight of every cell, FP32, for the frame's sensor panel
//                                          fv_up7_ducros_2d.cu.bak:393-428
__global__ void d2av_sensor_kernel(const GridDev gd, const double *buf, double sc, float *out)
{
    const int n = gd.n;
    const double h = gd.h;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < (long long)n * n;
         k += (long long)blockDim.x * gridDim.x) {
        const int j = (int)(k / n), i = (int)(k % n);
        const long long e = d2_at(gd, j, i);
        double p, c0, u, v;
        d2_prim(gd.gam, buf[e], buf[e + gd.plane], buf[e + 2 * gd.plane], buf[e + 3 * gd.plane], p, c0, u, v);
        const double wc[6] = {-1., 9., -45., 45., -9., 1.};
        const int wo[6] = {-3, -2, -1, 1, 2, 3};
        double du_dx = 0., dv_dy = 0.;
        for (int m = 0; m < 6; ++m) {
            const long long ex = e + wo[m], ey = e + (long long)wo[m] * gd.pitch;
            double rx = buf[ex], ry = buf[ey];
            rx = rx > 1e-14 ? rx : 1e-14;
            ry = ry > 1e-14 ? ry : 1e-14;
            du_dx += wc[m] * (buf[ex + gd.plane] / rx);
            dv_dy += wc[m] * (buf[ey + 2 * gd.plane] / ry);
        }
        du_dx /= 60. * h;
        dv_dy /= 60. * h;
        double div_u = du_dx + dv_dy;
        if (div_u > 0.) div_u = 0.;
        const double sos2 = (sc / (h * h)) * c0 * c0;
        out[k] = (float)((div_u * div_u) / (div_u * div_u + sos2 + 1e-40));
    }
}

int sm_count()
{
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

template <int ORDER>
cudaError_t launch_order(const GridDev &gd, int stage, int tiles, const D2Params &av, cudaStream_t s)
{
    constexpr size_t smem = D2Shape<ORDER>::SMEM;
    LaunchFacts f{};
    cudaError_t e = launch_facts((const void *)d2av_stage_kernel<ORDER>, DNT, smem, f);
    if (e != cudaSuccess) return e;
    const int cap = f.ctas_per_sm * f.sms;
    d2av_stage_kernel<ORDER><<<tiles < cap ? tiles : cap, DNT, smem, s>>>(gd, stage, tiles, av);
    return cudaGetLastError();
}

}  // namespace

int d2av_ghost(int order) { return std::max((order + 1) / 2, 3); }

void d2av_tiles(int n, int &tiles_x, int &tiles)
{
    tiles_x = (n + DTX - 1) / DTX;
    tiles = tiles_x * ((n + DTY - 1) / DTY);
}

cudaError_t d2av_launch_stage(const GridDev &gd, int order, int stage, int tiles, const D2Params &av,
                              cudaStream_t s)
{
    if (order == 3) return launch_order<3>(gd, stage, tiles, av, s);
    if (order == 5) return launch_order<5>(gd, stage, tiles, av, s);
    if (order == 7) return launch_order<7>(gd, stage, tiles, av, s);
    if (order == 9) return launch_order<9>(gd, stage, tiles, av, s);
    return cudaErrorInvalidValue;
}

cudaError_t d2av_lam_into(const GridDev &gd, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(&gd.ctrl->lam_acc, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    const long long n2 = (long long)gd.n * gd.n;
    const int blocks = (int)std::min<long long>((n2 + 255) / 256, 4LL * sm_count());
    d2av_lam_kernel<<<blocks, 256, 0, s>>>(gd, (const double *)gd.st[0]);
    return cudaGetLastError();
}

cudaError_t d2av_sensor_into(const GridDev &gd, double sc, float *out, cudaStream_t s)
{
    const long long n2 = (long long)gd.n * gd.n;
    const int blocks = (int)std::min<long long>((n2 + 255) / 256, 4LL * sm_count());
    d2av_sensor_kernel<<<blocks, 256, 0, s>>>(gd, (const double *)gd.st[0], sc, out);
    return cudaGetLastError();
}

}  // namespace fvb
