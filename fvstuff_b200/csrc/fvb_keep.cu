// fvb_keep.cu -- the KEEP flux family of keep_fv_euler_2d.cu on the device.
//
// Collocated FV on conserved cell averages (g = 2), FP64.  Per face:
//   F = F_EC + (1 - phi) F_JST + phi F_RH
// with F_EC the entropy-conserving / kinetic-energy-preserving central flux,
// F_JST a 4th-order background dissipation, F_RH the MOVERS-RH scalar
// dissipation, and phi in {0, 1} the entropy-distance shock sensor scaled by
// the stage input's global maximum (keep_fv_euler_2d.cu:145-369).
//
// That maximum must be known before any flux, so a stage is two launches:
// keep_ed_kernel (per-cell entropy distance, block max, atomicMax into the
// step control) and keep_stage_kernel (tile in shared memory, every face
// once, divergence, RK combination with floors, stores with ghost images,
// and in stage 3 the wave-speed max for the next dt).  Both convert each
// cell of a tile once -- floored primitives, entropy and entropy variables
// -- and form every face's terms from those, so no face repeats the
// divisions and logarithms of its two cells.  The step control is the same
// device-side Ctrl as the UP path.
#include "fvb_aux.h"
#include "fvb_physics.cuh"
#include "fvb_device.cuh"

namespace fvb {
namespace {

constexpr double KG_MIN = 1e-14;

__device__ __forceinline__ double k_snd(double rho, double p, double gam) { return sqrt(gam * p / rho); }

// floored primitives and entropy s = ln(p / rho^gamma) of a conserved cell
//                                              keep_fv_euler_2d.cu:99-132
__device__ __forceinline__ void k_cell(const double U[4], double gam, double W[4], double Uf[4], double &s)
{
    double rho = smax<double>(U[0], KG_MIN), mx = U[1], my = U[2], E = U[3];
    double u = mx / rho, v = my / rho;
    W[0] = rho;
    W[1] = mx / rho;
    W[2] = my / rho;
    W[3] = smax<double>((gam - 1.) * (E - 0.5 * rho * (u * u + v * v)), KG_MIN);
    Uf[0] = rho; Uf[1] = mx; Uf[2] = my; Uf[3] = E;
    s = log(W[3] / pow(W[0], gam));
}

// entropy variables from primitives and their entropy   keep_fv:123-132
__device__ __forceinline__ void k_evars(const double W[4], double s, double gam, double V[4])
{
    double rho = W[0], u = W[1], v = W[2], p = W[3];
    V[0] = (gam - s) / (gam - 1.) - rho * (u * u + v * v) / (2. * p);
    V[1] = rho * u / p;
    V[2] = rho * v / p;
    V[3] = -rho / p;
}

// ECKEP central flux (Cartesian) and MOVERS-RH coefficient  keep_fv:145-219
// VL, VR: the two cells' entropy variables in the face frame (the Cartesian
// ones of k_evars with (u, v) -> (un, ut): for the normals (1, 0) and (0, 1)
// a relabelling and one exact negation, so the values are the reference's)
//
// The steps and their association order are the published flux's as the
// reference evaluates them (the ECKEP averages, the MOVERS-RH coefficient
// with its division by dV3^2 + 1e-16 and the sonic fix), not a rewrite:
// where dV3 is small that division amplifies a last-bit difference in its
// operands by many orders of magnitude, so any reassociation here moves the
// low-Mach vortex run outside the spread between the reference's own GPU
// and host builds, which is the tolerance this family is held to.
__device__ __forceinline__ void k_flux(const double WL[4], const double WR[4], const double VL[4],
                                       const double VR[4], double nx, double ny, double gam, double Fec[4],
                                       double *alphaS)
{
    const double rL = WL[0], uL = WL[1], vL = WL[2], pL = WL[3];
    const double rR = WR[0], uR = WR[1], vR = WR[2], pR = WR[3];
    const double unL = uL * nx + vL * ny, utL = -uL * ny + vL * nx;
    const double unR = uR * nx + vR * ny, utR = -uR * ny + vR * nx;
    const double EL = pL / (gam - 1.) + 0.5 * rL * (unL * unL + utL * utL);
    const double ER = pR / (gam - 1.) + 0.5 * rR * (unR * unR + utR * utR);
    const double UL[4] = {rL, rL * unL, rL * utL, EL};
    const double UR[4] = {rR, rR * unR, rR * utR, ER};
    const double FL[4] = {rL * unL, rL * unL * unL + pL, rL * unL * utL, (EL + pL) * unL};
    const double FR[4] = {rR * unR, rR * unR * unR + pR, rR * unR * utR, (ER + pR) * unR};
    const double dV0 = VR[0] - VL[0], dV1 = VR[1] - VL[1], dV2 = VR[2] - VL[2], dV3 = VR[3] - VL[3];
    const double dpsi = rR * unR - rL * unL;
    const double Fc0 = 0.5 * (FL[0] + FR[0]);
    const double unb = 0.5 * (unL + unR), utb = 0.5 * (utL + utR), pb = 0.5 * (pL + pR);
    const double Fc1 = Fc0 * unb + pb;
    const double Fc2 = Fc0 * utb;
    const double Feb = 0.5 * (FL[3] + FR[3]);
    const double num = dV0 * Fc0 + dV1 * Fc1 + dV2 * Fc2 + dV3 * Feb - dpsi;
    const double Fc3 = Feb - (num / (dV3 * dV3 + 1e-16)) * dV3;
    Fec[0] = Fc0;
    Fec[1] = Fc1 * nx - Fc2 * ny;
    Fec[2] = Fc1 * ny + Fc2 * nx;
    Fec[3] = Fc3;
    const double rav = 0.5 * (rL + rR);
    const double aav = k_snd(smax<double>(rav, KG_MIN), smax<double>(pb, KG_MIN), gam);
    const double l1 = fabs(unb - aav), l2 = fabs(unb), l3 = fabs(unb + aav);
    const double lmin = smin<double>(l1, smin<double>(l2, l3)), lmax = smax<double>(l1, smax<double>(l2, l3));
    double aS = lmax;
    for (int q = 0; q < 4; ++q) {
        const double dU = UR[q] - UL[q];
        double sk;
        if (fabs(dU) < 1e-12) {
            sk = lmin;
        } else {
            sk = fabs((FR[q] - FL[q]) / dU);
            if (sk >= lmax) sk = lmax;
            else if (sk <= lmin) sk = lmin;
        }
        if (sk < aS) aS = sk;
    }
    if (aS < 0.1) aS = (aS * aS + 0.1 * 0.1) / (2. * 0.1);
    *alphaS = aS;
}

__device__ __forceinline__ void load_cell(const double *buf, const GridDev &gd, int j, int i, double U[4])
{
    long long e = (long long)(j + gd.g) * gd.pitch + (i + gd.g) + gd.xoff;
    for (int q = 0; q < 4; ++q) U[q] = buf[e + q * gd.plane];
}

struct KCtl {
    double dt;
    int run;
};

constexpr int KTX = 32, KTY = 16, KNT = 256, KG = 2;
constexpr int KSW = KTX + 2 * KG, KSH = KTY + 2 * KG, KPL = KSW * KSH;
constexpr int EW = KTX + 1, EH = KTY + 1, EPL = EW * EH;  // a tile and its right / top neighbours

// per-cell max of the entropy distance |(U_n - U_c) . (V_n - V_c)| across
// its right and top faces, max-reduced into ctrl->aux; a tile's cells and
// their right / top neighbours are converted once each (floored conserved
// state and entropy variables in shared memory)   keep_fv_euler_2d.cu:249-277
__global__ void __launch_bounds__(KNT) keep_ed_kernel(const GridDev gd, const double *buf, int ntiles)
{
    __shared__ double sU[4][EPL], sV[4][EPL];
    __shared__ double sh[KNT / 32];
    const int tid = threadIdx.x, n = gd.n;
    double m = 0.0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int tx0 = (t % gd.tiles_x) * KTX, ty0 = (t / gd.tiles_x) * KTY;
        for (int k = tid; k < EPL; k += KNT) {
            const int r = k / EW, c = k - r * EW, j = ty0 + r, i = tx0 + c;
            double U[4] = {1, 0, 0, 2.5};  // admissible filler beyond the ghost layer
            if (j <= n && i <= n) load_cell(buf, gd, j, i, U);
            double W[4], Uf[4], sc, V[4];
            k_cell(U, gd.gam, W, Uf, sc);
            k_evars(W, sc, gd.gam, V);
            for (int q = 0; q < 4; ++q) {
                sU[q][k] = Uf[q];
                sV[q][k] = V[q];
            }
        }
        __syncthreads();
        for (int k = tid; k < KTX * KTY; k += KNT) {
            const int r = k / KTX, c = k - r * KTX;
            if (ty0 + r >= n || tx0 + c >= n) continue;
            const int b = r * EW + c;
            double ex = 0., ey = 0.;
            for (int q = 0; q < 4; ++q) {
                ex += (sU[q][b + 1] - sU[q][b]) * (sV[q][b + 1] - sV[q][b]);
                ey += (sU[q][b + EW] - sU[q][b]) * (sV[q][b + EW] - sV[q][b]);
            }
            m = fmax(m, fmax(fabs(ex), fabs(ey)));
        }
        __syncthreads();
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((tid & 31) == 0) sh[tid >> 5] = m;
    __syncthreads();
    if (tid == 0) {
        double b = 0.0;
        for (int w = 0; w < KNT / 32; ++w) b = fmax(b, sh[w]);
        atomicMax(&gd.ctrl->aux, (unsigned long long)__double_as_longlong(b));
    }
}

// one SSP-RK3 stage of the KEEP scheme               keep_fv_euler_2d.cu:298-393
__global__ void __launch_bounds__(KNT, 2) keep_stage_kernel(const GridDev gd, int stage, int ntiles)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *U = reinterpret_cast<double *>(smem_raw);  // [4][KSH][KSW] conserved, rho floored
    double *W = U + 4 * KPL;                           // [4] floored primitives
    double *V = W + 4 * KPL;                           // [4] entropy variables (Cartesian)
    double *FX = V + 4 * KPL;                          // [4][KTY][KTX+1]
    double *FY = FX + 4 * KTY * (KTX + 1);             // [4][KTY+1][KTX]
    __shared__ KCtl s_ctl;
    __shared__ double s_red[KNT / 32];
    const int tid = threadIdx.x, n = gd.n, np = n + 2 * KG;
    const double gam = gd.gam;
    const double *in = (const double *)(stage == 2 ? gd.k1 : stage == 3 ? gd.k2 : gd.st[0]);
    const double *u0 = (const double *)gd.st[0];
    double *out = (double *)(stage == 1 ? gd.k1 : stage == 2 ? gd.k2 : gd.st[0]);
    const double edmax = __longlong_as_double((long long)gd.ctrl->aux);
    const double inv_h = 1. / gd.h;

    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int tx0 = (t % gd.tiles_x) * KTX, ty0 = (t / gd.tiles_x) * KTY;
        if (tid == 0) {
            TileCtl c = tile_control<P64>(gd.ctrl, stage, t == 0);
            s_ctl = KCtl{c.dt, c.run};
        }
        __syncthreads();
        const KCtl ctl = s_ctl;
        if (!ctl.run) {
            __syncthreads();
            continue;
        }
        for (int k = tid; k < KPL; k += KNT) {
            const int r = k / KSW, c = k - r * KSW, jp = ty0 + r, ip = tx0 + c;
            double Uc[4] = {1, 0, 0, 2.5};
            if (jp < np && ip < np) {
                long long e = (long long)jp * gd.pitch + ip + gd.xoff;
                for (int q = 0; q < 4; ++q) Uc[q] = in[e + q * gd.plane];
            }
            double Wc[4], Fc[4], sc, Vc[4];
            k_cell(Uc, gam, Wc, Fc, sc);
            k_evars(Wc, sc, gam, Vc);
            for (int q = 0; q < 4; ++q) {
                U[q * KPL + k] = Fc[q];
                W[q * KPL + k] = Wc[q];
                V[q * KPL + k] = Vc[q];
            }
        }
        __syncthreads();
        // faces: x then y; the face lies between cells a (left/bottom) and
        // b = a + st, with the JST stencil reaching a - st and b + st
        for (int f = tid; f < (KTX + 1) * KTY + KTX * (KTY + 1); f += KNT) {
            const bool xf = f < (KTX + 1) * KTY;
            int r, c, st;
            if (xf) { r = f / (KTX + 1); c = f - r * (KTX + 1); st = 1; }
            else { const int f2 = f - (KTX + 1) * KTY; r = f2 / KTX; c = f2 - r * KTX; st = KSW; }
            const int b = (r + KG) * KSW + (c + KG), a = b - st;
            const double nx = xf ? 1. : 0., ny = xf ? 0. : 1.;
            double WL[4], WR[4], UL[4], UR[4], Up2[4], Um1[4], VL[4], VR[4], fec[4], aS;
            for (int q = 0; q < 4; ++q) {
                WL[q] = W[q * KPL + a]; WR[q] = W[q * KPL + b];
                UL[q] = U[q * KPL + a]; UR[q] = U[q * KPL + b];
                Up2[q] = U[q * KPL + b + st]; Um1[q] = U[q * KPL + a - st];
                VL[q] = V[q * KPL + a]; VR[q] = V[q * KPL + b];
            }
            // face frame: (un, ut) = (u, v) on x-faces, (v, -u) on y-faces
            const double VLn[4] = {VL[0], xf ? VL[1] : VL[2], xf ? VL[2] : -VL[1], VL[3]};
            const double VRn[4] = {VR[0], xf ? VR[1] : VR[2], xf ? VR[2] : -VR[1], VR[3]};
            k_flux(WL, WR, VLn, VRn, nx, ny, gam, fec, &aS);
            const double unL = WL[1] * nx + WL[2] * ny, unR = WR[1] * nx + WR[2] * ny;
            const double aR = k_snd(0.5 * (WL[0] + WR[0]), 0.5 * (WL[3] + WR[3]), gam);
            const double lamt = smax<double>(fabs(unL), fabs(unR)) + aR;
            const double aJST = (1.0 / 32.0) * lamt;
            // entropy distance of the face                  keep_fv:249-258
            double ed = 0.;
            for (int q = 0; q < 4; ++q) ed += (UR[q] - UL[q]) * (VR[q] - VL[q]);
            const double sed = fabs(ed) / (edmax + 1e-30);
            const double phi = (1. - exp(-12.0 * sed)) > 0.05 ? 1. : 0.;
            double *o = xf ? FX + r * (KTX + 1) + c : FY + r * KTX + c;
            const int os = xf ? KTY * (KTX + 1) : (KTY + 1) * KTX;
            for (int q = 0; q < 4; ++q) {
                const double jst = aJST * (Up2[q] - 3. * UR[q] + 3. * UL[q] - Um1[q]);
                const double rh = -0.5 * aS * (UR[q] - UL[q]);
                o[q * os] = fec[q] + (1. - phi) * jst + phi * rh;
            }
        }
        __syncthreads();
        double lmax = 0.0;
        for (int k = tid; k < KTX * KTY; k += KNT) {
            const int r = k / KTX, c = k - r * KTX, i = tx0 + c, j = ty0 + r;
            if (i >= n || j >= n) continue;
            const long long e = (long long)(j + KG) * gd.pitch + (i + KG) + gd.xoff;
            double v[4];
            for (int q = 0; q < 4; ++q) {
                const double *fx = FX + q * KTY * (KTX + 1) + r * (KTX + 1) + c;
                const double *fy = FY + q * (KTY + 1) * KTX + r * KTX + c;
                const double L = -(fx[1] - fx[0] + fy[KTX] - fy[0]) * inv_h;
                const double ua = u0[e + q * gd.plane];  // U0
                const double ub = in[e + q * gd.plane];  // stage input (U0, U1 or U2)
                if (stage == 1) v[q] = 1. * ua + 0. * ua + 1. * ctl.dt * L;
                else if (stage == 2) v[q] = 0.75 * ua + 0.25 * ub + 0.25 * ctl.dt * L;
                else v[q] = (1. / 3.) * ua + (2. / 3.) * ub + (2. / 3.) * ctl.dt * L;
            }
            v[0] = smax<double>(v[0], KG_MIN);
            v[3] = smax<double>(v[3], KG_MIN);
            put_cell<double>(gd, out, j, i, v);
            if (stage == 3) {
                double Wn[4], Fn[4], sn;
                k_cell(v, gam, Wn, Fn, sn);
                const double cs = k_snd(Wn[0], Wn[3], gam);
                lmax = smax<double>((fabs(Wn[1]) + cs) + (fabs(Wn[2]) + cs), lmax);
            }
        }
        if (stage == 3) {
            for (int o = 16; o > 0; o >>= 1) lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
            if ((tid & 31) == 0) s_red[tid >> 5] = lmax;
            __syncthreads();
            if (tid == 0) {
                double m = 0.0;
                for (int w = 0; w < KNT / 32; ++w) m = fmax(m, s_red[w]);
                atomicMax(&gd.ctrl->lam_acc, (unsigned long long)__double_as_longlong(m));
                if (t == 0) leader_finish<P64>(gd.ctrl);
            }
        }
        __syncthreads();
    }
}

// (|u| + c) + (|v| + c) of a conserved state, max into ctrl->lam_acc
__global__ void keep_lam_kernel(const GridDev gd)
{
    __shared__ double sh[32];
    const int n = gd.n;
    const long long n2 = (long long)n * n;
    double m = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n2;
         k += (long long)blockDim.x * gridDim.x) {
        double U[4], W[4], Fc[4], s;
        load_cell((const double *)gd.st[0], gd, (int)(k / n), (int)(k % n), U);
        k_cell(U, gd.gam, W, Fc, s);
        const double cs = k_snd(W[0], W[3], gd.gam);
        m = fmax(m, (fabs(W[1]) + cs) + (fabs(W[2]) + cs));
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

size_t keep_smem() { return sizeof(double) * (12 * KPL + 4 * KTY * (KTX + 1) + 4 * (KTY + 1) * KTX); }

}  // namespace

void keep_tiles(int n, int &tiles_x, int &tiles)
{
    tiles_x = (n + KTX - 1) / KTX;
    tiles = tiles_x * ((n + KTY - 1) / KTY);
}

// one KEEP stage: clear the sensor max, the entropy-distance pass, then the
// fused flux / RK / ghost kernel
cudaError_t keep_launch_stage(const GridDev &gd, int stage, int tiles, cudaStream_t s)
{
    LaunchFacts f{};
    cudaError_t e = launch_facts((const void *)keep_stage_kernel, KNT, keep_smem(), f);
    if (e != cudaSuccess) return e;
    const int ctas_per_sm = f.ctas_per_sm, sms = f.sms;
    const void *in = stage == 2 ? gd.k1 : stage == 3 ? gd.k2 : gd.st[0];
    e = cudaMemsetAsync(&gd.ctrl->aux, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    const int eb = tiles < 4 * sms ? tiles : 4 * sms;
    keep_ed_kernel<<<eb, KNT, 0, s>>>(gd, (const double *)in, tiles);
    const int grid = tiles < ctas_per_sm * sms ? tiles : ctas_per_sm * sms;
    keep_stage_kernel<<<grid, KNT, keep_smem(), s>>>(gd, stage, tiles);
    return cudaGetLastError();
}

cudaError_t keep_lam_into(const GridDev &gd, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(&gd.ctrl->lam_acc, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    int blocks = (int)(((long long)gd.n * gd.n + 255) / 256);
    if (blocks > 1184) blocks = 1184;
    keep_lam_kernel<<<blocks, 256, 0, s>>>(gd);
    return cudaGetLastError();
}

}  // namespace fvb
