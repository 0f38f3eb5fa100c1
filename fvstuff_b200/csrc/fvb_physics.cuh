// fvb_physics.cuh -- pointwise physics and face numerics of the UP-ORDER +
// Ducros-blended HLLC/HLLE finite-volume Euler step, for the device.
//
// Everything works in the face-normal frame: a state is (rho, un, ut, p)
// with un the velocity along the face normal and ut the tangential one, and
// a flux comes back as (mass, normal momentum, tangential momentum, energy).
// An x-face takes (u, v) as (un, ut); a y-face takes (v, u) and the caller
// swaps the two momentum components back.  For the unit normals the
// reference uses, (1,0) and (0,1), this relabelling is exactly its rotation
// (fv_up7_ducros_2d.cu:245-248, :287-290).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fvb {

// Literal of type R spelled as the reference spells it (1.4f in the FP32
// solver, 1.4 in the FP64 one), so constants round identically.
#define FVB_LIT(R, x) (sizeof(R) == 4 ? R(x##f) : R(x))

template <class R> __device__ __forceinline__ R dsqrt(R x);
template <> __device__ __forceinline__ float dsqrt<float>(float x) { return sqrtf(x); }
template <> __device__ __forceinline__ double dsqrt<double>(double x) { return sqrt(x); }
template <class R> __device__ __forceinline__ R dmin(R a, R b);
template <> __device__ __forceinline__ float dmin<float>(float a, float b) { return fminf(a, b); }
template <> __device__ __forceinline__ double dmin<double>(double a, double b) { return fmin(a, b); }
template <class R> __device__ __forceinline__ R dmax(R a, R b);
template <> __device__ __forceinline__ float dmax<float>(float a, float b) { return fmaxf(a, b); }
template <> __device__ __forceinline__ double dmax<double>(double a, double b) { return fmax(a, b); }
template <class R> __device__ __forceinline__ R dabs(R a);
template <> __device__ __forceinline__ float dabs<float>(float a) { return fabsf(a); }
template <> __device__ __forceinline__ double dabs<double>(double a) { return fabs(a); }

// Min / max as one compare and a select, for the FP64 throughput paths.  An
// FP64 fmin / fmax is not one instruction on sm_100: with its NaN rules it
// issues about 7.5 (a compare, selects, integer and bit operations; ncu
// op-class counters of a loop of them), a compare and a select 3.  smax(a, b)
// is a > b ? a : b, smin(a, b) is a < b ? a : b: for finite operands the
// value fmax / fmin give (up to the sign of a zero result), and with a
// constant second operand (the clamps at 0, 1e-10, 1e-14) for every first
// operand, NaN included (NaN -> the constant).  FP32 keeps fminf / fmaxf,
// one instruction.
template <class R> __device__ __forceinline__ R smin(R a, R b);
template <> __device__ __forceinline__ float smin<float>(float a, float b) { return fminf(a, b); }
template <> __device__ __forceinline__ double smin<double>(double a, double b) { return a < b ? a : b; }
template <class R> __device__ __forceinline__ R smax(R a, R b);
template <> __device__ __forceinline__ float smax<float>(float a, float b) { return fmaxf(a, b); }
template <> __device__ __forceinline__ double smax<double>(double a, double b) { return a > b ? a : b; }

// floor used on reconstructed and updated rho and p: x > c ? x : c, so a
// NaN becomes the floor (fv_up7_ducros_2d.cu:421-422, :543-544); the same
// value as fmax(x, c) for every input
template <class R> __device__ __forceinline__ R floor14(R x)
{
    return smax<R>(x, FVB_LIT(R, 1e-14));
}

// Gas constants of one solver.  gm1 is formed as gamma - 1 at run time, the
// same subtraction the reference performs on its GAMMA_V literal.
template <class R> struct Gas {
    R gam, gm1;
};

// c = sqrt(max(gamma p / rho, 1e-14))           fv_up7_ducros_2d.cu:63-68
template <class R> __device__ __forceinline__ R sound(R p, R rho, const Gas<R> &gs)
{
    R cs2 = gs.gam * p / rho;
    const R c = FVB_LIT(R, 1e-14);
    return dsqrt<R>(cs2 > c ? cs2 : c);
}

// total energy of a primitive state            fv_up7_ducros_2d.cu:77, :251
template <class R> __device__ __forceinline__ R etot(R r, R a, R b, R p, const Gas<R> &gs)
{
    return p / gs.gm1 + FVB_LIT(R, 0.5) * r * (a * a + b * b);
}

// primitive <-> conserved                      fv_up7_ducros_2d.cu:71-88
template <class R> __device__ __forceinline__ void p2c(const R w[4], R c[4], const Gas<R> &gs)
{
    c[0] = w[0];
    c[1] = w[0] * w[1];
    c[2] = w[0] * w[2];
    c[3] = etot(w[0], w[1], w[2], w[3], gs);
}
template <class R> __device__ __forceinline__ void c2p(const R c[4], R w[4], const Gas<R> &gs)
{
    w[0] = c[0];
    w[1] = c[1] / c[0];
    w[2] = c[2] / c[0];
    w[3] = gs.gm1 * (c[3] - FVB_LIT(R, 0.5) * (c[1] * c[1] + c[2] * c[2]) / c[0]);
}

// pressure-jump sensor s = dp^2 / (dp^2 + 0.1 (pa+pb)^2)
//                                               fv_up7_ducros_2d.cu:114-133
template <class R> __device__ __forceinline__ R ducros(R pa, R pb)
{
    R dp = pb - pa, ps = pb + pa;
    return dp * dp / (dp * dp + FVB_LIT(R, 0.1) * ps * ps);
}

// Upwind-biased face values from the 2g-point stencil s[0..2g-1] along the
// normal (the face lies between s[g-1] and s[g]); arithmetic in RR, result
// rounded to R.                                 fv_up7_ducros_2d.cu:149-186
template <class R, class RR, int ORDER>
__device__ __forceinline__ void upface(const R *s, R &vL, R &vR)
{
    if constexpr (ORDER == 3) {
        vL = R((-RR(s[0]) + RR(5.0) * s[1] + RR(2.0) * s[2]) / RR(6.0));
        vR = R((RR(2.0) * s[1] + RR(5.0) * s[2] - RR(s[3])) / RR(6.0));
    } else if constexpr (ORDER == 5) {
        vL = R((RR(2.0) * s[0] - RR(13.0) * s[1] + RR(47.0) * s[2] + RR(27.0) * s[3] - RR(3.0) * s[4]) / RR(60.0));
        vR = R((-RR(3.0) * s[1] + RR(27.0) * s[2] + RR(47.0) * s[3] - RR(13.0) * s[4] + RR(2.0) * s[5]) / RR(60.0));
    } else if constexpr (ORDER == 9) {
        // the published UP9 weights, as they stand (the left-biased set sums
        // to 4217/2520, not one)                 fv_up7_ducros_2d.cu:176-186
        vL = R((RR(3.0) * s[0] - RR(25.0) * s[1] + RR(101.0) * s[2] - RR(319.0) * s[3] + RR(2765.0) * s[4]
                + RR(2139.0) * s[5] - RR(533.0) * s[6] + RR(97.0) * s[7] - RR(11.0) * s[8]) / RR(2520.0));
        vR = R((-RR(11.0) * s[1] + RR(97.0) * s[2] - RR(533.0) * s[3] + RR(2139.0) * s[4] + RR(2765.0) * s[5]
                - RR(319.0) * s[6] + RR(101.0) * s[7] - RR(25.0) * s[8] + RR(3.0) * s[9]) / RR(2520.0));
    } else {
        static_assert(ORDER == 7, "ORDER must be 3, 5, 7 or 9");
        vL = R((-RR(3.0) * s[0] + RR(25.0) * s[1] - RR(101.0) * s[2] + RR(319.0) * s[3]
                + RR(214.0) * s[4] - RR(38.0) * s[5] + RR(4.0) * s[6]) / RR(420.0));
        vR = R((RR(4.0) * s[1] - RR(38.0) * s[2] + RR(214.0) * s[3] + RR(319.0) * s[4]
                - RR(101.0) * s[5] + RR(25.0) * s[6] - RR(3.0) * s[7]) / RR(420.0));
    }
}

// total energy of a normal-frame state with the kinetic term summed in the
// Cartesian order u^2 + v^2, as the reference sums it for every face: for a
// y-face (YF) the normal component is v, so the tangential square comes
// first (the two orders round differently under a fused multiply-add)
template <bool YF, class R>
__device__ __forceinline__ R etot_cart(R r, R un, R ut, R p, const Gas<R> &gs)
{
    return YF ? etot(r, ut, un, p, gs) : etot(r, un, ut, p, gs);
}

// HLLC with Davis wave-speed bounds, normal frame (YF: a y-face)
//                                               fv_up7_ducros_2d.cu:237-292
template <class R, bool YF = false>
__device__ __forceinline__ void hllc(const R L[4], const R Rr[4], R F[4], const Gas<R> &gs)
{
    R rL = L[0], uL = L[1], tL = L[2], pL = L[3];
    R rR = Rr[0], uR = Rr[1], tR = Rr[2], pR = Rr[3];
    R cL = sound(pL, rL, gs), cR = sound(pR, rR, gs);
    R EL = etot_cart<YF>(rL, uL, tL, pL, gs), ER = etot_cart<YF>(rR, uR, tR, pR, gs);
    R SL = dmin<R>(uL - cL, uR - cR);
    R SR = dmax<R>(uL + cL, uR + cR);
    const R zero = R(0);
    if (SL >= zero) {
        F[0] = rL * uL; F[1] = rL * uL * uL + pL; F[2] = rL * uL * tL; F[3] = (EL + pL) * uL;
        return;
    }
    if (SR <= zero) {
        F[0] = rR * uR; F[1] = rR * uR * uR + pR; F[2] = rR * uR * tR; F[3] = (ER + pR) * uR;
        return;
    }
    R dL = rL * (SL - uL), dR = rR * (SR - uR);
    R Ss = (pR - pL + dL * uL - dR * uR) / (dL - dR);
    bool left = (Ss >= zero);
    R rK = left ? rL : rR, uK = left ? uL : uR, tK = left ? tL : tR;
    R pK = left ? pL : pR, EK = left ? EL : ER, SK = left ? SL : SR;
    R fact = rK * (SK - uK) / (SK - Ss);
    R Us1 = fact * Ss, Us2 = fact * tK;
    R Us3 = fact * (EK / rK + (Ss - uK) * (Ss + pK / (rK * (SK - uK))));
    F[0] = rK * uK + SK * (fact - rK);
    F[1] = rK * uK * uK + pK + SK * (Us1 - rK * uK);
    F[2] = rK * uK * tK + SK * (Us2 - rK * tK);
    F[3] = (EK + pK) * uK + SK * (Us3 - EK);
}

// HLLE on the two adjacent cell averages, normal frame (YF: a y-face)
//                                               fv_up7_ducros_2d.cu:296-328
template <class R, bool YF = false>
__device__ __forceinline__ void hlle(const R L[4], const R Rr[4], R F[4], const Gas<R> &gs)
{
    R rL = L[0], uL = L[1], tL = L[2], pL = L[3];
    R rR = Rr[0], uR = Rr[1], tR = Rr[2], pR = Rr[3];
    R cL = sound(pL, rL, gs), cR = sound(pR, rR, gs);
    R EL = etot_cart<YF>(rL, uL, tL, pL, gs), ER = etot_cart<YF>(rR, uR, tR, pR, gs);
    R FL0 = rL * uL, FL1 = rL * uL * uL + pL, FL2 = rL * uL * tL, FL3 = (EL + pL) * uL;
    R FR0 = rR * uR, FR1 = rR * uR * uR + pR, FR2 = rR * uR * tR, FR3 = (ER + pR) * uR;
    R SL = dmin<R>(uL - cL, uR - cR);
    R SR = dmax<R>(uL + cL, uR + cR);
    const R zero = R(0);
    if (SL >= zero) { F[0] = FL0; F[1] = FL1; F[2] = FL2; F[3] = FL3; return; }
    if (SR <= zero) { F[0] = FR0; F[1] = FR1; F[2] = FR2; F[3] = FR3; return; }
    R dS = dmax<R>(SR - SL, FVB_LIT(R, 1e-10));
    R SRL = SR * SL;
    F[0] = (SR * FL0 - SL * FR0 + SRL * (rR - rL)) / dS;
    F[1] = (SR * FL1 - SL * FR1 + SRL * (rR * uR - rL * uL)) / dS;
    F[2] = (SR * FL2 - SL * FR2 + SRL * (rR * tR - rL * tL)) / dS;
    F[3] = (SR * FL3 - SL * FR3 + SRL * (ER - EL)) / dS;
}

// ===========================================================================
// Division-free forms for the throughput paths (FP64 plain and FP32c).  The
// same formulas as above, with each quotient written as a product with one
// reciprocal, the reciprocals shared where the reference divides by the same
// quantity twice, 1/(gamma-1) precomputed, and the cell-centred sound speed
// and energy of the HLLE states taken from per-cell values computed once.
// Results differ from the reference's association order by a few ulp.
// ===========================================================================

// Reciprocal and square root per arithmetic type.  Every argument on these
// paths is a positive normal number (densities and pressures are floored at
// 1e-14, wave-speed spans at 1e-10, sound speeds squared at 1e-14).
//
// FP64 reciprocal: the hardware seed (rcp.approx.ftz.f64, relative error
// 2^-19.9 measured) and one third-order Newton-Raphson step,
//   e = 1 - x y,  y' = y (1 + e + e^2),
// whose error is O(e^3) ~ 2^-60 before the last rounding (a higher-order
// Newton-Raphson iteration for 1/x, as in Muller et al., Handbook of
// Floating-Point Arithmetic).  Measured on B200 against the correctly
// rounded 1/x over 4M log-uniform samples in [1e-14, 1e14]: at most 1 ulp,
// 0.03% of samples not exact.  FVB_EXACT_RCP_SQRT=1 selects the correctly
// rounded library forms instead.
//
// FP64 square root: the hardware reciprocal-root seed (rsqrt.approx.ftz.f64,
// 2^-20.0 measured), one third-order step y' = y (1 + e/2 + 3e^2/8) with
// e = 1 - x y^2, then s = x y' and the residual correction
// s' = s + (x - s^2) y'/2 (the Newton step for sqrt through the reciprocal
// root, as in Markstein, IA-64 and Elementary Functions).  Measured: equal to the correctly rounded sqrt on all 4M samples.
//
// FP32: the hardware approximations (rcp / rsqrt, about 2 ulp).
#ifndef FVB_EXACT_RCP_SQRT
#define FVB_EXACT_RCP_SQRT 0
#endif
#if FVB_EXACT_RCP_SQRT
__device__ __forceinline__ double frcp(double x) { return __drcp_rn(x); }
__device__ __forceinline__ double fsqrt(double x) { return sqrt(x); }
#else
__device__ __forceinline__ double frcp(double x)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x, y, 1.0);
    return fma(y, fma(e, e, e), y);
}
__device__ __forceinline__ double fsqrt(double x)
{
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-(x * y), y, 1.0);
    y = fma(y, e * fma(e, 0.375, 0.5), y);
    const double s = x * y;
    return fma(fma(-s, s, x), 0.5 * y, s);
}
#endif
__device__ __forceinline__ float frcp(float x) { return __fdividef(1.0f, x); }
__device__ __forceinline__ float fsqrt(float x) { return x * rsqrtf(x); }

// FP64 sound speed c = sqrt(max(gp / r, 1e-14)) from gp = gamma p and the
// density, as gp / sqrt(gp r) = gp * rsqrt(gp r): the reciprocal root (seed
// and the third-order step of fsqrt) replaces a reciprocal of r and a
// square root; within 2 ulp of the correctly rounded sqrt(gp / r).  The
// floor test gp > 1e-14 r is cs2 > 1e-14 without the division (r > 0).
// sqrt(gp / r) without the floor (gp, r >= 1e-14)
__device__ __forceinline__ double snd_rsq_raw(double gp, double r)
{
#if FVB_EXACT_RCP_SQRT
    return sqrt(gp / r);
#else
    const double x = gp * r;
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-(x * y), y, 1.0);
    y = fma(y, e * fma(e, 0.375, 0.5), y);
    return gp * y;
#endif
}
// (both sides evaluated and one selected: no branch)
__device__ __forceinline__ double snd_rsq(double gp, double r)
{
    const double c = snd_rsq_raw(gp, r);
    return gp > 1e-14 * r ? c : 1e-7;
}

template <class R> struct GasF {
    R gam, igm1, gm1;  // gamma, 1/(gamma-1), gamma-1
};

// UP-ORDER face values with the weights pre-divided by their denominator
template <class R, int ORDER>
__device__ __forceinline__ void upface_fast(const R *s, R &vL, R &vR)
{
    if constexpr (ORDER == 3) {
        const R k = R(1.0 / 6.0);
        vL = (-s[0] + R(5) * s[1] + R(2) * s[2]) * k;
        vR = (R(2) * s[1] + R(5) * s[2] - s[3]) * k;
    } else if constexpr (ORDER == 5) {
        const R k = R(1.0 / 60.0);
        vL = (R(2) * s[0] - R(13) * s[1] + R(47) * s[2] + R(27) * s[3] - R(3) * s[4]) * k;
        vR = (-R(3) * s[1] + R(27) * s[2] + R(47) * s[3] - R(13) * s[4] + R(2) * s[5]) * k;
    } else if constexpr (ORDER == 9) {
#define FVB_W9(a) R((a) / 2520.0)
        vL = FVB_W9(3.) * s[0] + FVB_W9(-25.) * s[1] + FVB_W9(101.) * s[2] + FVB_W9(-319.) * s[3]
             + FVB_W9(2765.) * s[4] + FVB_W9(2139.) * s[5] + FVB_W9(-533.) * s[6] + FVB_W9(97.) * s[7]
             + FVB_W9(-11.) * s[8];
        vR = FVB_W9(-11.) * s[1] + FVB_W9(97.) * s[2] + FVB_W9(-533.) * s[3] + FVB_W9(2139.) * s[4]
             + FVB_W9(2765.) * s[5] + FVB_W9(-319.) * s[6] + FVB_W9(101.) * s[7] + FVB_W9(-25.) * s[8]
             + FVB_W9(3.) * s[9];
#undef FVB_W9
    } else {
        // weights pre-divided: one multiply and six fused multiply-adds a side
#define FVB_W7(a) R((a) / 420.0)
        vL = FVB_W7(-3.) * s[0] + FVB_W7(25.) * s[1] + FVB_W7(-101.) * s[2] + FVB_W7(319.) * s[3]
             + FVB_W7(214.) * s[4] + FVB_W7(-38.) * s[5] + FVB_W7(4.) * s[6];
        vR = FVB_W7(4.) * s[1] + FVB_W7(-38.) * s[2] + FVB_W7(214.) * s[3] + FVB_W7(319.) * s[4]
             + FVB_W7(-101.) * s[5] + FVB_W7(25.) * s[6] + FVB_W7(-3.) * s[7];
#undef FVB_W7
    }
}

// sound speed and total energy of a cell state (rho, a, b, p)
template <class R>
__device__ __forceinline__ void cell_ce(R r, R a, R b, R p, const GasF<R> &gs, R &c, R &E)
{
    if constexpr (sizeof(R) == 8) {
        c = snd_rsq(gs.gam * p, r);
    } else {
        R cs2 = gs.gam * p * frcp(r);
        c = fsqrt(cs2 > FVB_LIT(R, 1e-14) ? cs2 : FVB_LIT(R, 1e-14));
    }
    E = p * gs.igm1 + R(0.5) * r * (a * a + b * b);
}

// Blended face flux, normal frame: (1-s) HLLC(L, R) + s HLLE(WL, WR) with
// s the pressure-jump sensor of the two cells.  L, Rv: floored UP
// reconstructions; WL, WR: cell states with their sound speeds cW* and
// energies EW*.                               fv_up7_ducros_2d.cu:237-328, :433
//
// RS selects the solver on the reconstructed states: 0 HLLC (fv_up7), 1 HLL,
// 2 Roe with the Harten-Hyman entropy fix (carb_fv_2d.cu:116-211, the
// riemann_n alternatives of carb_fv), always blended with the HLLE of the
// cell states by the Ducros sensor.
template <class R>
__device__ __forceinline__ void hll_fast(const R L[4], const R Rv[4], const GasF<R> &gs, R Fh[4])
{
    const R zero = R(0);
    const R rL = L[0], uL = L[1], tL = L[2], pL = L[3];
    const R rR = Rv[0], uR = Rv[1], tR = Rv[2], pR = Rv[3];
    // sound speed without a floor, as carb_fv_2d.cu:60-61 (rho, p >= 1e-14)
    const R cL = snd_rsq_raw(gs.gam * pL, rL), cR = snd_rsq_raw(gs.gam * pR, rR);
    const R EL = pL * gs.igm1 + R(0.5) * rL * (uL * uL + tL * tL);
    const R ER = pR * gs.igm1 + R(0.5) * rR * (uR * uR + tR * tR);
    // Einfeldt's form of the two-wave average: FL, FR or the subsonic
    // average without selects
    const R SL = smin<R>(smin<R>(uL - cL, uR - cR), zero), SR = smax<R>(smax<R>(uL + cL, uR + cR), zero);
    const R inv = frcp(SR - SL), SRL = SR * SL;
    const R mL = rL * uL, mR = rR * uR;
    Fh[0] = (SR * mL - SL * mR + SRL * (rR - rL)) * inv;
    Fh[1] = (SR * (mL * uL + pL) - SL * (mR * uR + pR) + SRL * (mR - mL)) * inv;
    Fh[2] = (SR * (mL * tL) - SL * (mR * tR) + SRL * (rR * tR - rL * tL)) * inv;
    Fh[3] = (SR * ((EL + pL) * uL) - SL * ((ER + pR) * uR) + SRL * (ER - EL)) * inv;
}

template <class R>
__device__ __forceinline__ void roe_fast(const R L[4], const R Rv[4], const GasF<R> &gs, R Fh[4])
{
    const R zero = R(0);
    const R rL = L[0], uL = L[1], tL = L[2], pL = L[3];
    const R rR = Rv[0], uR = Rv[1], tR = Rv[2], pR = Rv[3];
    const R ip = frcp(rL * rR);
    const R irL = rR * ip, irR = rL * ip;
    const R cL = fsqrt(gs.gam * pL * irL), cR = fsqrt(gs.gam * pR * irR);
    const R sqL = fsqrt(rL), sqR = fsqrt(rR);
    const R iden = frcp(sqL + sqR);
    const R a = (sqL * uL + sqR * uR) * iden, b = (sqL * tL + sqR * tR) * iden;  // Roe normal / tangential velocity
    const R EL = pL * gs.igm1 + R(0.5) * rL * (uL * uL + tL * tL);
    const R ER = pR * gs.igm1 + R(0.5) * rR * (uR * uR + tR * tR);
    const R H = (sqL * ((EL + pL) * irL) + sqR * ((ER + pR) * irR)) * iden;
    const R c2 = gs.gm1 * (H - R(0.5) * (a * a + b * b));
    const R c = fsqrt(c2 > FVB_LIT(R, 1e-14) ? c2 : FVB_LIT(R, 1e-14));
    const R ic2 = frcp(c2);
    const R drho = rR - rL, dun = uR - uL, dut = tR - tL, dp = pR - pL;
    const R rr = sqL * sqR;
    const R b1 = (dp - rr * c * dun) * (R(0.5) * ic2);
    const R b2 = drho - dp * ic2;
    const R b3 = rr * dut;
    const R b4 = (dp + rr * c * dun) * (R(0.5) * ic2);
    // Harten-Hyman: |lambda| below eps/2 replaced by (lambda^2 + eps^2/4)/eps
    const R lam1 = a - c, lam4 = a + c;
    const R eps1 = smax<R>(R(2) * ((uR - cR) - (uL - cL)), zero);
    const R eps4 = smax<R>(R(2) * ((uR + cR) - (uL + cL)), zero);
    R al1 = dabs<R>(lam1), al4 = dabs<R>(lam4);
    const R al2 = dabs<R>(a);
    al1 = al1 < eps1 * R(0.5) ? (lam1 * lam1 + eps1 * eps1 * R(0.25)) * frcp(eps1) : al1;
    al4 = al4 < eps4 * R(0.5) ? (lam4 * lam4 + eps4 * eps4 * R(0.25)) * frcp(eps4) : al4;
    const R w1 = al1 * b1, w2 = al2 * b2, w3 = al2 * b3, w4 = al4 * b4;
    const R d0 = w1 + w2 + w4;
    const R d1 = w1 * lam1 + w2 * a + w4 * lam4;
    const R d2 = (w1 + w2 + w4) * b + w3;
    const R d3 = w1 * (H - a * c) + w2 * R(0.5) * (a * a + b * b) + w3 * b + w4 * (H + a * c);
    const R mL = rL * uL, mR = rR * uR;
    Fh[0] = R(0.5) * (mL + mR - d0);
    Fh[1] = R(0.5) * (mL * uL + pL + mR * uR + pR - d1);
    Fh[2] = R(0.5) * (mL * tL + mR * tR - d2);
    Fh[3] = R(0.5) * ((EL + pL) * uL + (ER + pR) * uR - d3);
}

// Solver on the reconstructed states (normal frame): HLLC, or with RS 1 / 2
// carb_fv's HLL / Roe.  Branch-free, so its chain can interleave with the
// HLLE chain where both are evaluated together.
template <class R, int RS = 0>
__device__ __forceinline__ void recon_flux_fast(const R L[4], const R Rv[4], const GasF<R> &gs, R Fh[4])
{
    const R zero = R(0);
    if constexpr (RS == 1 || RS == 2) {
        if constexpr (RS == 1) hll_fast<R>(L, Rv, gs, Fh);
        else roe_fast<R>(L, Rv, gs, Fh);
    } else {
        const R rL = L[0], uL = L[1], tL = L[2], pL = L[3];
        const R rR = Rv[0], uR = Rv[1], tR = Rv[2], pR = Rv[3];
        R cL, cR;
        if constexpr (sizeof(R) == 8) {
            // no reciprocal of the densities: c = gamma p rsqrt(gamma p rho)
            cL = snd_rsq(gs.gam * pL, rL);
            cR = snd_rsq(gs.gam * pR, rR);
        } else {
            const R cs2L = gs.gam * pL * frcp(rL), cs2R = gs.gam * pR * frcp(rR);
            cL = fsqrt(cs2L > FVB_LIT(R, 1e-14) ? cs2L : FVB_LIT(R, 1e-14));
            cR = fsqrt(cs2R > FVB_LIT(R, 1e-14) ? cs2R : FVB_LIT(R, 1e-14));
        }
        const R SL = smin<R>(uL - cL, uR - cR), SR = smax<R>(uL + cL, uR + cR);
        const R dL = rL * (SL - uL), dR = rR * (SR - uR);
        const R Ss = (pR - pL + dL * uL - dR * uR) * frcp(dL - dR);
        // side K: by the contact when subsonic, by the fan when supersonic
        const bool supL = (SL >= zero);
        const bool sup = supL || (SR <= zero);
        const bool left = sup ? supL : (Ss >= zero);
        const R rK = left ? rL : rR, uK = left ? uL : uR, tK = left ? tL : tR;
        const R pK = left ? pL : pR, SK = left ? SL : SR;
        const R dK = left ? dL : dR;
        // only side K's energy enters the flux: one evaluation, after the
        // selection (the same expression as for either side)
        const R EK = pK * gs.igm1 + R(0.5) * rK * (uK * uK + tK * tK);
        // star terms weighted by SK, or by 0 when supersonic (q forced
        // finite), so one set of expressions gives both fluxes.  With
        // dK = rK (SK - uK) and q = 1 / (SK - Ss):  fact = dK q, and
        //   fact (EK / rK + (Ss - uK)(Ss + pK / dK))
        //     = q (EK (SK - uK) + (Ss - uK)(dK Ss + pK))   (no 1/rK, no 1/dK);
        // the tangential momentum flux is the mass flux times tK
        const R SKw = sup ? zero : SK;
        const R q = sup ? zero : frcp(SK - Ss);
        const R fact = dK * q;
        const R m = rK * uK;
        Fh[0] = m + SKw * (fact - rK);
        Fh[1] = m * uK + pK + SKw * (fact * Ss - m);
        Fh[2] = Fh[0] * tK;
        Fh[3] = (EK + pK) * uK + SKw * (q * (EK * (SK - uK) + (Ss - uK) * (dK * Ss + pK)) - EK);
    }
}

// HLLE of the two cell states (sound speeds cWL, cWR, energies EWL, EWR) and
// the pressure-jump sensor s of the face, normal frame.
template <class R>
__device__ __forceinline__ void hlle_sensor_fast(const R WL[4], const R WR[4], R cWL, R cWR, R EWL, R EWR, R Fl[4],
                                                 R &sd)
{
    const R zero = R(0);
    const R rL = WL[0], uL = WL[1], tL = WL[2], pL = WL[3];
    const R rR = WR[0], uR = WR[1], tR = WR[2], pR = WR[3];
    // Einfeldt's form: with SL- = min(SL, 0), SR+ = max(SR, 0) the HLL
    // average equals FL, FR or the subsonic average in the three wave
    // configurations, with no selects
    const R SL = smin<R>(smin<R>(uL - cWL, uR - cWR), zero), SR = smax<R>(smax<R>(uL + cWL, uR + cWR), zero);
    const R mL = rL * uL, mR = rR * uR;
    const R FL1 = mL * uL + pL, FR1 = mR * uR + pR;
    const R FL2 = mL * tL, FR2 = mR * tR;
    const R FL3 = (EWL + pL) * uL, FR3 = (EWR + pR) * uR;
    const R dS = smax<R>(SR - SL, FVB_LIT(R, 1e-10));
    const R dp = WR[3] - WL[3], ps = WR[3] + WL[3];
    const R dp2 = dp * dp;
    const R dd = dp2 + FVB_LIT(R, 0.1) * ps * ps;
    R idS;
    if constexpr (sizeof(R) == 8) {
        // one FP64 reciprocal for the HLLE span and the sensor's
        // denominator (dS >= 1e-10, dd >= 4e-29: the product is normal)
        const R ip = frcp(dS * dd);
        idS = dd * ip;
        sd = dp2 * (dS * ip);
    } else {
        idS = frcp(dS);
        sd = dp2 * frcp(dd);
    }
    const R SRL = SR * SL;
    Fl[0] = (SR * mL - SL * mR + SRL * (rR - rL)) * idS;
    Fl[1] = (SR * FL1 - SL * FR1 + SRL * (mR - mL)) * idS;
    Fl[2] = (SR * FL2 - SL * FR2 + SRL * (rR * tR - rL * tL)) * idS;
    Fl[3] = (SR * FL3 - SL * FR3 + SRL * (EWR - EWL)) * idS;
}

// Ducros blend (1 - s) Fh + s Fl
template <class R>
__device__ __forceinline__ void ducros_blend(const R Fh[4], const R Fl[4], R sd, R F[4])
{
#pragma unroll
    for (int q = 0; q < 4; ++q) F[q] = Fh[q] + sd * (Fl[q] - Fh[q]);
}

template <class R, int RS = 0>
__device__ __forceinline__ void face_flux_fast(const R L[4], const R Rv[4], const R WL[4], const R WR[4], R cWL,
                                               R cWR, R EWL, R EWR, const GasF<R> &gs, R F[4])
{
    R Fh[4], Fl[4], sd;
    recon_flux_fast<R, RS>(L, Rv, gs, Fh);
    hlle_sensor_fast<R>(WL, WR, cWL, cWR, EWL, EWR, Fl, sd);
    ducros_blend<R>(Fh, Fl, sd, F);
}

}  // namespace fvb
