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

// floor used on reconstructed and updated rho and p (x > c ? x : c, so a
// NaN becomes the floor, as in fv_up7_ducros_2d.cu:421-422, :543-544)
template <class R> __device__ __forceinline__ R floor14(R x)
{
    const R c = FVB_LIT(R, 1e-14);
    return x > c ? x : c;
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
    } else {
        static_assert(ORDER == 7, "ORDER must be 3, 5 or 7");
        vL = R((-RR(3.0) * s[0] + RR(25.0) * s[1] - RR(101.0) * s[2] + RR(319.0) * s[3]
                + RR(214.0) * s[4] - RR(38.0) * s[5] + RR(4.0) * s[6]) / RR(420.0));
        vR = R((RR(4.0) * s[1] - RR(38.0) * s[2] + RR(214.0) * s[3] + RR(319.0) * s[4]
                - RR(101.0) * s[5] + RR(25.0) * s[6] - RR(3.0) * s[7]) / RR(420.0));
    }
}

// HLLC with Davis wave-speed bounds, normal frame
//                                               fv_up7_ducros_2d.cu:237-292
template <class R>
__device__ __forceinline__ void hllc(const R L[4], const R Rr[4], R F[4], const Gas<R> &gs)
{
    R rL = L[0], uL = L[1], tL = L[2], pL = L[3];
    R rR = Rr[0], uR = Rr[1], tR = Rr[2], pR = Rr[3];
    R cL = sound(pL, rL, gs), cR = sound(pR, rR, gs);
    R EL = etot(rL, uL, tL, pL, gs), ER = etot(rR, uR, tR, pR, gs);
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

// HLLE on the two adjacent cell averages, normal frame
//                                               fv_up7_ducros_2d.cu:296-328
template <class R>
__device__ __forceinline__ void hlle(const R L[4], const R Rr[4], R F[4], const Gas<R> &gs)
{
    R rL = L[0], uL = L[1], tL = L[2], pL = L[3];
    R rR = Rr[0], uR = Rr[1], tR = Rr[2], pR = Rr[3];
    R cL = sound(pL, rL, gs), cR = sound(pR, rR, gs);
    R EL = etot(rL, uL, tL, pL, gs), ER = etot(rR, uR, tR, pR, gs);
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

}  // namespace fvb
