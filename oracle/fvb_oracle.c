/*
 * fvb_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * Plain-C restatement of fvStuff's finite-volume Euler step, used by the
 * tests as the parity checker and by bench.py as the timed CPU baseline.
 * The product library never links it.  Built by oracle/Makefile with
 * -ffp-contract=off so that every operation rounds once, as written.
 *
 *   fvb_oracle_up7.h  : UP-ORDER + Ducros HLLC/HLLE path (fv_up7_ducros_2d.cu),
 *                       instantiated in float (as shipped) and double
 *   fvb_oracle_keep.h : ECKEP + JST/MOVERS-RH path (keep_fv_euler_2d.cu), double
 *   fvb_oracle_rec3.h : rec3 + HLLC + 2x2-block Zhang-Shu path (fv_rec3_2d.cu), double
 *   fvb_oracle_d2av.h : UP + HLLC + Ducros-gated D2 viscosity path
 *                       (fv_up7_ducros_2d.cu.bak), double
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

/* ---- single precision instantiation ------------------------------------ */
#define REAL float
#define OSFX(n) n##_f32
#define RL(x) x##f
#define OSQRT sqrtf
#define OFABS fabsf
#define OFMIN fminf
#define OFMAX fmaxf
#define OTANH tanhf
#include "fvb_oracle_up7.h"
#undef REAL
#undef OSFX
#undef RL
#undef OSQRT
#undef OFABS
#undef OFMIN
#undef OFMAX
#undef OTANH

/* ---- double precision instantiation ------------------------------------ */
#define REAL double
#define OSFX(n) n##_f64
#define RL(x) x
#define OSQRT sqrt
#define OFABS fabs
#define OFMIN fmin
#define OFMAX fmax
#define OTANH tanh
#include "fvb_oracle_up7.h"

#include "fvb_oracle_keep.h"

#include "fvb_oracle_rec3.h"

#include "fvb_oracle_d2av.h"

/* ---- single-face entry points (unit tests of the Riemann solvers) ------- */
void orc_hllc_f64(const double L[4], const double R[4], double F[4]) { hllc_f64(L, R, F); }
void orc_hlle_f64(const double L[4], const double R[4], double F[4]) { hlle_f64(L, R, F); }
void orc_hllc_f32(const float L[4], const float R[4], float F[4]) { hllc_f32(L, R, F); }
void orc_hlle_f32(const float L[4], const float R[4], float F[4]) { hlle_f32(L, R, F); }
void orc_hll_f64(const double L[4], const double R[4], double F[4]) { hll_f64(L, R, F); }
void orc_roe_f64(const double L[4], const double R[4], double F[4]) { roe_f64(L, R, F); }
void orc_upface_f64(int order, const double *s, double *vL, double *vR) { upface_f64(order, s, vL, vR); }
void orc_upface_f32(int order, const float *s, float *vL, float *vR) { upface_f32(order, s, vL, vR); }
void orc_d2av_hllc(const double L[4], const double R[4], double F[4]) { d2_hllc(L, R, F); }
