// fvb_face2.cuh -- the FP32 face flux of the compensated form, evaluated for
// two faces at once in the packed FP32 pairs of sm_100 (FFMA2 / FADD2 /
// FMUL2: one instruction issues the same operation on both halves of a
// 64-bit register pair).  Lane x and lane y are two independent faces; every
// operation below acts on both, so the arithmetic of two faces issues as one
// instruction stream.  Per-lane work (reciprocals, square roots, compares,
// selects, min / max) stays scalar.
//
// The scheme is the reference's UP7 + Ducros-blended HLLC / HLLE face flux
// (fv_up7_ducros_2d.cu:149-186, :237-328, :433), normal frame, written for
// FP32 throughput:
//   * UP7 weights pre-divided by 420;
//   * HLLC: one side K (the upwind side of the contact, or the upwind side of
//     the whole fan when it is supersonic) is selected once; the star terms
//     are added with weight SK, or 0 when supersonic, so the supersonic and
//     subsonic fluxes come out of the same expressions; the star energy uses
//     q = 1/(SK - S*) only:  fact (EK/rK + (S*-uK)(S* + pK/dK))
//                          = q (EK (SK - uK) + (S*-uK)(dK S* + pK)),
//     with dK = rK (SK - uK), and the tangential momentum flux is the mass
//     flux times uK_t;
//   * HLLE (Einfeldt's form): with SL- = min(SL, 0) and SR+ = max(SR, 0),
//     (SR+ FL - SL- FR + SR+ SL- (UR - UL)) / (SR+ - SL-) equals FL, FR or the
//     HLL average in the three wave configurations, with no selects;
//   * blend F = Fh + s (Fl - Fh), s the pressure-jump sensor.
// Each rewriting is exact in real arithmetic; in FP32 the results differ from
// the reference's association order by a few ulp, which the compensated
// form's tolerance against the FP64 oracle (1e-6 relative L1) absorbs.
#pragma once
#include <cuda_runtime.h>

#include "fvb_physics.cuh"

namespace fvb {
namespace f2 {

typedef float2 V;

__device__ __forceinline__ V splat(float a) { return make_float2(a, a); }
__device__ __forceinline__ V add(V a, V b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ V mul(V a, V b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ V fma(V a, V b, V c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ V sub(V a, V b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
// a * b - c
__device__ __forceinline__ V fms(V a, V b, V c) { return __ffma2_rn(a, b, make_float2(-c.x, -c.y)); }
__device__ __forceinline__ V vmin(V a, V b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }
__device__ __forceinline__ V vmax(V a, V b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
__device__ __forceinline__ V rcp(V a) { return make_float2(__fdividef(1.0f, a.x), __fdividef(1.0f, a.y)); }
// sqrt of x >= 1e-14 as x * rsqrt(x)
__device__ __forceinline__ V vsqrt(V a) { return mul(a, make_float2(rsqrtf(a.x), rsqrtf(a.y))); }

struct B {
    bool x, y;
};
__device__ __forceinline__ V sel(B c, V a, V b) { return make_float2(c.x ? a.x : b.x, c.y ? a.y : b.y); }

// UP7 face values of a pair of 8-point stencils (face between s[3] and s[4])
__device__ __forceinline__ void upface7(const V s[8], V &vL, V &vR)
{
#define FVB_W7(a) splat((float)((a) / 420.0))
    vL = mul(FVB_W7(-3.), s[0]);
    vL = fma(FVB_W7(25.), s[1], vL);
    vL = fma(FVB_W7(-101.), s[2], vL);
    vL = fma(FVB_W7(319.), s[3], vL);
    vL = fma(FVB_W7(214.), s[4], vL);
    vL = fma(FVB_W7(-38.), s[5], vL);
    vL = fma(FVB_W7(4.), s[6], vL);
    vR = mul(FVB_W7(4.), s[1]);
    vR = fma(FVB_W7(-38.), s[2], vR);
    vR = fma(FVB_W7(214.), s[3], vR);
    vR = fma(FVB_W7(319.), s[4], vR);
    vR = fma(FVB_W7(-101.), s[5], vR);
    vR = fma(FVB_W7(25.), s[6], vR);
    vR = fma(FVB_W7(-3.), s[7], vR);
#undef FVB_W7
}

// Blended flux of two faces, normal frame.  L, Rv: floored reconstructions
// (rho, un, ut, p); WL, WR: the cell states either side with their sound
// speeds cWL, cWR and energies EWL, EWR.
__device__ __forceinline__ void face_flux(const V L[4], const V Rv[4], const V WL[4], const V WR[4], V cWL,
                                          V cWR, V EWL, V EWR, float gam, float igm1, V F[4])
{
    const V zero = splat(0.0f), half = splat(0.5f), G = splat(gam), IG = splat(igm1);
    const V tiny = splat(1e-14f);
    // --- HLLC of the reconstructed states ---
    V Fh0, Fh1, Fh2, Fh3;
    {
        const V rL = L[0], uL = L[1], tL = L[2], pL = L[3];
        const V rR = Rv[0], uR = Rv[1], tR = Rv[2], pR = Rv[3];
        const V cL = vsqrt(vmax(mul(mul(G, pL), rcp(rL)), tiny));
        const V cR = vsqrt(vmax(mul(mul(G, pR), rcp(rR)), tiny));
        const V SL = vmin(sub(uL, cL), sub(uR, cR)), SR = vmax(add(uL, cL), add(uR, cR));
        const V dL = mul(rL, sub(SL, uL)), dR = mul(rR, sub(SR, uR));
        const V Ss = mul(sub(fma(dL, uL, sub(pR, pL)), mul(dR, uR)), rcp(sub(dL, dR)));
        // side K: by the contact when subsonic, by the fan when supersonic
        const B supL{SL.x >= 0.0f, SL.y >= 0.0f};
        const B sup{supL.x || SR.x <= 0.0f, supL.y || SR.y <= 0.0f};
        const B left{sup.x ? supL.x : Ss.x >= 0.0f, sup.y ? supL.y : Ss.y >= 0.0f};
        const V rK = sel(left, rL, rR), uK = sel(left, uL, uR), tK = sel(left, tL, tR);
        const V pK = sel(left, pL, pR), SK = sel(left, SL, SR);
        const V dK = sel(left, dL, dR);
        // only side K's energy enters the flux: one evaluation, after the selection
        const V EK = fma(mul(half, rK), fma(uK, uK, mul(tK, tK)), mul(pK, IG));
        // star weight: SK when subsonic, 0 when supersonic (q forced finite)
        const V SKw = sel(sup, zero, SK);
        const V q = sel(sup, zero, rcp(sub(SK, Ss)));
        const V fact = mul(dK, q);
        const V m = mul(rK, uK);
        Fh0 = fma(SKw, sub(fact, rK), m);
        Fh1 = fma(SKw, fms(fact, Ss, m), fma(m, uK, pK));
        Fh2 = mul(Fh0, tK);
        const V e3 = fma(EK, sub(SK, uK), mul(sub(Ss, uK), fma(dK, Ss, pK)));
        Fh3 = fma(SKw, fms(q, e3, EK), mul(add(EK, pK), uK));
    }
    // --- HLLE of the cell states (Einfeldt form), and the sensor ---
    V Fl0, Fl1, Fl2, Fl3, sd;
    {
        const V rL = WL[0], uL = WL[1], tL = WL[2], pL = WL[3];
        const V rR = WR[0], uR = WR[1], tR = WR[2], pR = WR[3];
        const V SLm = vmin(vmin(sub(uL, cWL), sub(uR, cWR)), zero);
        const V SRp = vmax(vmax(add(uL, cWL), add(uR, cWR)), zero);
        const V mL = mul(rL, uL), mR = mul(rR, uR);
        const V idS = rcp(vmax(sub(SRp, SLm), splat(1e-10f)));
        const V SRL = mul(SRp, SLm);
        Fl0 = mul(fma(SRL, sub(rR, rL), fms(SRp, mL, mul(SLm, mR))), idS);
        Fl1 = mul(fma(SRL, sub(mR, mL), fms(SRp, fma(mL, uL, pL), mul(SLm, fma(mR, uR, pR)))), idS);
        Fl2 = mul(fma(SRL, fms(rR, tR, mul(rL, tL)), fms(SRp, mul(mL, tL), mul(SLm, mul(mR, tR)))), idS);
        Fl3 = mul(fma(SRL, sub(EWR, EWL), fms(SRp, mul(add(EWL, pL), uL), mul(SLm, mul(add(EWR, pR), uR)))),
                  idS);
        const V dp = sub(pR, pL), ps = add(pR, pL);
        const V dp2 = mul(dp, dp);
        sd = mul(dp2, rcp(fma(mul(splat(0.1f), ps), ps, dp2)));
    }
    // --- Ducros blend ---
    F[0] = fma(sd, sub(Fl0, Fh0), Fh0);
    F[1] = fma(sd, sub(Fl1, Fh1), Fh1);
    F[2] = fma(sd, sub(Fl2, Fh2), Fh2);
    F[3] = fma(sd, sub(Fl3, Fh3), Fh3);
}

}  // namespace f2
}  // namespace fvb
