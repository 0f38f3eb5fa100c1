/*
 * fvb_oracle_up7.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * CPU restatement of the UP-ORDER + Ducros-blended HLLC/HLLE finite-volume
 * Euler step of fvStuff's fv_up7_ducros_2d.cu.  Only the tests, the smoke
 * check and the CPU-baseline leg of bench.py load this code; the product
 * (libfvb.so) never links or calls it.
 *
 * This body is included twice by fvb_oracle.c:
 *   REAL   = float  -> the solver as shipped (FP32 state, FP64 reconstruction
 *                      arithmetic rounded to float, as fv_up7_ducros_2d.cu:152-185)
 *   REAL   = double -> the FP64 form of the same solver
 * with OSFX(name) appending the precision suffix and RL(x) spelling a literal
 * of type REAL (1.4f vs 1.4) so every constant rounds exactly as the
 * reference's literals do.
 *
 * Arithmetic is written with the reference's association order so that,
 * compiled without FMA contraction, it is bit-identical to the reference's
 * own kernels compiled for the host (checked by tests/test_oracle_pin.py).
 *
 * Layout: padded SoA, Q[q*Np*Np + jp*Np + ip], Np = N + 2g, interior cell
 * (j,i) at (jp,ip) = (j+g, i+g)            -- fv_up7_ducros_2d.cu:49-56
 */

/* ---- pointwise physics ------------------------------------------------- */

/* c = sqrt(max(gamma p / rho, 1e-14))          fv_up7_ducros_2d.cu:63-68 */
static inline REAL OSFX(snd)(REAL p, REAL rho)
{
    REAL cs2 = RL(1.4) * p / rho;
    return OSQRT(cs2 > RL(1e-14) ? cs2 : RL(1e-14));
}

/* total energy of a primitive state; the same expression is used by
 * p2c (fv_up7:77), hllc_n (:251-252) and hlle_n (:308-309)              */
static inline REAL OSFX(etot)(REAL r, REAL a, REAL b, REAL p)
{
    return p / (RL(1.4) - RL(1.)) + RL(0.5) * r * (a * a + b * b);
}

/* primitive -> conserved                        fv_up7_ducros_2d.cu:71-78 */
static inline void OSFX(p2c)(const REAL w[4], REAL c[4])
{
    c[0] = w[0];
    c[1] = w[0] * w[1];
    c[2] = w[0] * w[2];
    c[3] = OSFX(etot)(w[0], w[1], w[2], w[3]);
}

/* conserved -> primitive                        fv_up7_ducros_2d.cu:81-88 */
static inline void OSFX(c2p)(const REAL c[4], REAL w[4])
{
    w[0] = c[0];
    w[1] = c[1] / c[0];
    w[2] = c[2] / c[0];
    w[3] = (RL(1.4) - RL(1.)) * (c[3] - RL(0.5) * (c[1] * c[1] + c[2] * c[2]) / c[0]);
}

/* pressure-jump face sensor s = dp^2/(dp^2 + 0.1 (pL+pR)^2)
 *                                               fv_up7_ducros_2d.cu:114-133 */
static inline REAL OSFX(ducros)(REAL pa, REAL pb)
{
    REAL dp = pb - pa, ps = pb + pa;
    return dp * dp / (dp * dp + RL(0.1) * ps * ps);
}

/* ---- upwind-biased face values, FP64 arithmetic -------------------------
 * s[] holds the stencil along the face normal; the face sits between
 * s[g-1] and s[g].  vL is the left-biased value, vR the right-biased one.
 *                                               fv_up7_ducros_2d.cu:149-186 */
static inline void OSFX(upface)(int order, const REAL *s, REAL *vL, REAL *vR)
{
    double a0 = s[0], a1 = s[1], a2 = s[2], a3 = s[3];
    if (order == 3) {
        *vL = (REAL)((-a0 + 5.0 * a1 + 2.0 * a2) / 6.0);
        *vR = (REAL)((2.0 * a1 + 5.0 * a2 - a3) / 6.0);
        return;
    }
    double a4 = s[4], a5 = s[5];
    if (order == 5) {
        *vL = (REAL)((2.0 * a0 - 13.0 * a1 + 47.0 * a2 + 27.0 * a3 - 3.0 * a4) / 60.0);
        *vR = (REAL)((-3.0 * a1 + 27.0 * a2 + 47.0 * a3 - 13.0 * a4 + 2.0 * a5) / 60.0);
        return;
    }
    double a6 = s[6], a7 = s[7];
    if (order == 9) {
        /* the reference's UP9 weights are reproduced as published in the
         * solver; their left-biased set does not sum to one             */
        double a8 = s[8], a9 = s[9];
        *vL = (REAL)((3.0 * a0 - 25.0 * a1 + 101.0 * a2 - 319.0 * a3 + 2765.0 * a4
                      + 2139.0 * a5 - 533.0 * a6 + 97.0 * a7 - 11.0 * a8) / 2520.0);
        *vR = (REAL)((-11.0 * a1 + 97.0 * a2 - 533.0 * a3 + 2139.0 * a4 + 2765.0 * a5
                      - 319.0 * a6 + 101.0 * a7 - 25.0 * a8 + 3.0 * a9) / 2520.0);
        return;
    }
    *vL = (REAL)((-3.0 * a0 + 25.0 * a1 - 101.0 * a2 + 319.0 * a3
                  + 214.0 * a4 - 38.0 * a5 + 4.0 * a6) / 420.0);
    *vR = (REAL)((4.0 * a1 - 38.0 * a2 + 214.0 * a3 + 319.0 * a4
                  - 101.0 * a5 + 25.0 * a6 - 3.0 * a7) / 420.0);
}

/* ---- Riemann fluxes in the face-normal frame ----------------------------
 * States are (rho, un, ut, p) with un the face-normal and ut the tangential
 * velocity; fluxes come back as (mass, normal mom., tangential mom., energy).
 * An x-face is (u, v) -> (un, ut); a y-face is (v, u) -> (un, ut) with the
 * two momentum components swapped back by the caller.  For the unit normals
 * (1,0) and (0,1) the reference's rotations (fv_up7:245-248, :287-290) reduce
 * to exactly this relabelling, so the results are the same bits.          */

/* HLLC with Davis wave-speed bounds             fv_up7_ducros_2d.cu:237-292 */
static void OSFX(hllc)(const REAL L[4], const REAL R[4], REAL F[4])
{
    REAL rL = L[0], uL = L[1], tL = L[2], pL = L[3];
    REAL rR = R[0], uR = R[1], tR = R[2], pR = R[3];
    REAL cL = OSFX(snd)(pL, rL), cR = OSFX(snd)(pR, rR);
    REAL EL = OSFX(etot)(rL, uL, tL, pL);
    REAL ER = OSFX(etot)(rR, uR, tR, pR);
    REAL SL = OFMIN(uL - cL, uR - cR);
    REAL SR = OFMAX(uL + cL, uR + cR);
    if (SL >= RL(0.0)) {
        F[0] = rL * uL; F[1] = rL * uL * uL + pL; F[2] = rL * uL * tL; F[3] = (EL + pL) * uL;
        return;
    }
    if (SR <= RL(0.0)) {
        F[0] = rR * uR; F[1] = rR * uR * uR + pR; F[2] = rR * uR * tR; F[3] = (ER + pR) * uR;
        return;
    }
    REAL dL = rL * (SL - uL), dR = rR * (SR - uR);
    REAL Ss = (pR - pL + dL * uL - dR * uR) / (dL - dR);
    int left = (Ss >= RL(0.0));
    REAL rK = left ? rL : rR, uK = left ? uL : uR, tK = left ? tL : tR;
    REAL pK = left ? pL : pR, EK = left ? EL : ER, SK = left ? SL : SR;
    REAL fact = rK * (SK - uK) / (SK - Ss);
    REAL Us0 = fact;
    REAL Us1 = fact * Ss;
    REAL Us2 = fact * tK;
    REAL Us3 = fact * (EK / rK + (Ss - uK) * (Ss + pK / (rK * (SK - uK))));
    F[0] = rK * uK + SK * (Us0 - rK);
    F[1] = rK * uK * uK + pK + SK * (Us1 - rK * uK);
    F[2] = rK * uK * tK + SK * (Us2 - rK * tK);
    F[3] = (EK + pK) * uK + SK * (Us3 - EK);
}

/* HLLE                                          fv_up7_ducros_2d.cu:296-328 */
static void OSFX(hlle)(const REAL L[4], const REAL R[4], REAL F[4])
{
    REAL rL = L[0], uL = L[1], tL = L[2], pL = L[3];
    REAL rR = R[0], uR = R[1], tR = R[2], pR = R[3];
    REAL cL = OSFX(snd)(pL, rL), cR = OSFX(snd)(pR, rR);
    REAL EL = OSFX(etot)(rL, uL, tL, pL);
    REAL ER = OSFX(etot)(rR, uR, tR, pR);
    REAL UL[4] = { rL, rL * uL, rL * tL, EL };
    REAL UR[4] = { rR, rR * uR, rR * tR, ER };
    REAL FL[4] = { rL * uL, rL * uL * uL + pL, rL * uL * tL, (EL + pL) * uL };
    REAL FR[4] = { rR * uR, rR * uR * uR + pR, rR * uR * tR, (ER + pR) * uR };
    REAL SL = OFMIN(uL - cL, uR - cR);
    REAL SR = OFMAX(uL + cL, uR + cR);
    if (SL >= RL(0.0)) { for (int q = 0; q < 4; q++) F[q] = FL[q]; return; }
    if (SR <= RL(0.0)) { for (int q = 0; q < 4; q++) F[q] = FR[q]; return; }
    REAL dS = OFMAX(SR - SL, RL(1e-10));
    for (int q = 0; q < 4; q++)
        F[q] = (SR * FL[q] - SL * FR[q] + SR * SL * (UR[q] - UL[q])) / dS;
}

/* ---- Riemann-solver variants of carb_fv_2d.cu, normal frame ------------
 * (The reference's rotation by n = (1,0) or (0,1) reduces to the same
 * relabelling as above; for (0,1) its tangential velocity is -u, which only
 * flips the sign of the tangential terms and is undone by its back-rotation,
 * exactly, since negation is exact.)  Sound speed as carb_fv_2d.cu:60-61,
 * without the 1e-14 floor of fv_up7.                                        */
static inline REAL OSFX(snd_carb)(REAL rho, REAL p) { return OSQRT(RL(1.4) * p / rho); }

/* HLL, two waves with Davis bounds             carb_fv_2d.cu:116-150 */
static void OSFX(hll)(const REAL L[4], const REAL R[4], REAL F[4])
{
    REAL rL = L[0], uL = L[1], tL = L[2], pL = L[3];
    REAL rR = R[0], uR = R[1], tR = R[2], pR = R[3];
    REAL cL = OSFX(snd_carb)(rL, pL), cR = OSFX(snd_carb)(rR, pR);
    REAL EL = OSFX(etot)(rL, uL, tL, pL), ER = OSFX(etot)(rR, uR, tR, pR);
    REAL SL = OFMIN(uL - cL, uR - cR);
    REAL SR = OFMAX(uL + cL, uR + cR);
    REAL FL[4] = { rL * uL, rL * uL * uL + pL, rL * uL * tL, (EL + pL) * uL };
    REAL FR[4] = { rR * uR, rR * uR * uR + pR, rR * uR * tR, (ER + pR) * uR };
    if (SL >= RL(0.)) { for (int q = 0; q < 4; q++) F[q] = FL[q]; return; }
    if (SR <= RL(0.)) { for (int q = 0; q < 4; q++) F[q] = FR[q]; return; }
    REAL UL[4] = { rL, rL * uL, rL * tL, EL };
    REAL UR[4] = { rR, rR * uR, rR * tR, ER };
    REAL inv = RL(1.) / (SR - SL);
    for (int q = 0; q < 4; q++) F[q] = (SR * FL[q] - SL * FR[q] + SL * SR * (UR[q] - UL[q])) * inv;
}

/* Roe with the Harten-Hyman entropy fix        carb_fv_2d.cu:153-211 */
static void OSFX(roe)(const REAL L[4], const REAL R[4], REAL F[4])
{
    REAL rL = L[0], uL = L[1], tL = L[2], pL = L[3];
    REAL rR = R[0], uR = R[1], tR = R[2], pR = R[3];
    REAL cL = OSFX(snd_carb)(rL, pL), cR = OSFX(snd_carb)(rR, pR);
    REAL sqL = OSQRT(rL), sqR = OSQRT(rR);
    REAL den = sqL + sqR;
    REAL aRoe = (sqL * uL + sqR * uR) / den;   /* normal velocity      */
    REAL bRoe = (sqL * tL + sqR * tR) / den;   /* tangential velocity  */
    REAL HL = (pL / (RL(1.4) - RL(1.)) + RL(0.5) * rL * (uL * uL + tL * tL) + pL) / rL;
    REAL HR = (pR / (RL(1.4) - RL(1.)) + RL(0.5) * rR * (uR * uR + tR * tR) + pR) / rR;
    REAL HRoe = (sqL * HL + sqR * HR) / den;
    REAL c2 = (RL(1.4) - RL(1.)) * (HRoe - RL(0.5) * (aRoe * aRoe + bRoe * bRoe));
    REAL cRoe = OSQRT(c2 > RL(1e-14) ? c2 : RL(1e-14));
    REAL EL = OSFX(etot)(rL, uL, tL, pL), ER = OSFX(etot)(rR, uR, tR, pR);
    REAL FL[4] = { rL * uL, rL * uL * uL + pL, rL * uL * tL, (EL + pL) * uL };
    REAL FR[4] = { rR * uR, rR * uR * uR + pR, rR * uR * tR, (ER + pR) * uR };
    REAL drho = rR - rL, dun = uR - uL, dut = tR - tL, dp = pR - pL;
    REAL rRoe = sqL * sqR;
    REAL b1 = (dp - rRoe * cRoe * dun) / (RL(2.) * c2);
    REAL b2 = drho - dp / c2;
    REAL b3 = rRoe * dut;
    REAL b4 = (dp + rRoe * cRoe * dun) / (RL(2.) * c2);
    REAL lam1 = aRoe - cRoe, lam2 = aRoe, lam3 = aRoe, lam4 = aRoe + cRoe;
    REAL eps1 = OFMAX(RL(0.), RL(2.) * ((uR - cR) - (uL - cL)));
    REAL eps4 = OFMAX(RL(0.), RL(2.) * ((uR + cR) - (uL + cL)));
    REAL al1 = OFABS(lam1);
    if (al1 < eps1 * RL(0.5)) al1 = (lam1 * lam1 + eps1 * eps1 * RL(0.25)) / eps1;
    REAL al2 = OFABS(lam2), al3 = OFABS(lam3);
    REAL al4 = OFABS(lam4);
    if (al4 < eps4 * RL(0.5)) al4 = (lam4 * lam4 + eps4 * eps4 * RL(0.25)) / eps4;
    REAL d0 = al1 * b1 + al2 * b2 + al4 * b4;
    REAL d1 = al1 * b1 * (aRoe - cRoe) + al2 * b2 * aRoe + al4 * b4 * (aRoe + cRoe);
    REAL d2 = al1 * b1 * bRoe + al2 * b2 * bRoe + al3 * b3 + al4 * b4 * bRoe;
    REAL d3 = al1 * b1 * (HRoe - aRoe * cRoe) + al2 * b2 * RL(0.5) * (aRoe * aRoe + bRoe * bRoe)
            + al3 * b3 * bRoe + al4 * b4 * (HRoe + aRoe * cRoe);
    F[0] = RL(0.5) * (FL[0] + FR[0]) - RL(0.5) * d0;
    F[1] = RL(0.5) * (FL[1] + FR[1]) - RL(0.5) * d1;
    F[2] = RL(0.5) * (FL[2] + FR[2]) - RL(0.5) * d2;
    F[3] = RL(0.5) * (FL[3] + FR[3]) - RL(0.5) * d3;
}

/* Blended face flux between the cells at offsets -1 and 0 of a stencil
 * gathered along the normal (stride st from base index b):
 *   F = (1-s) HLLC(UP recon) + s HLLE(cell averages)
 * comp[] maps (rho,u,v,p) slots to the normal frame: {0,1,2,3} for x-faces,
 * {0,2,1,3} for y-faces.                       fv_up7_ducros_2d.cu:414-494 */
static void OSFX(face)(const REAL *Q, size_t Np2, ptrdiff_t b, ptrdiff_t st,
                       int order, int rs, const int comp[4], REAL F[4])
{
    int g = (order + 1) / 2;
    REAL s[10], L[4], R[4], WL[4], WR[4], Fh[4], Fl[4];
    for (int q = 0; q < 4; q++) {
        const REAL *v = Q + (size_t)comp[q] * Np2;
        for (int d = 0; d < 2 * g; d++) s[d] = v[b + (ptrdiff_t)(d - g) * st];
        OSFX(upface)(order, s, &L[q], &R[q]);
        WL[q] = v[b - st];
        WR[q] = v[b];
    }
    L[0] = L[0] > RL(1e-14) ? L[0] : RL(1e-14);
    R[0] = R[0] > RL(1e-14) ? R[0] : RL(1e-14);
    L[3] = L[3] > RL(1e-14) ? L[3] : RL(1e-14);
    R[3] = R[3] > RL(1e-14) ? R[3] : RL(1e-14);
    /* rs: the solver on the reconstructed states -- 0 HLLC (fv_up7), 1 HLL,
     * 2 Roe (carb_fv_2d.cu's riemann_n choices) */
    if (rs == 1) OSFX(hll)(L, R, Fh);
    else if (rs == 2) OSFX(roe)(L, R, Fh);
    else OSFX(hllc)(L, R, Fh);
    OSFX(hlle)(WL, WR, Fl);
    REAL sd = OSFX(ducros)(WL[3], WR[3]);
    REAL Fn[4];
    for (int q = 0; q < 4; q++) Fn[q] = (RL(1.0) - sd) * Fh[q] + sd * Fl[q];
    for (int q = 0; q < 4; q++) F[comp[q]] = Fn[q];
}

/* ---- grid operators ---------------------------------------------------- */

/* Residual dU/dt = -(dF/dx + dG/dy) of the conserved variables and the cell
 * spectral radius |u|+|v|+c.  Q: padded primitives; RHS: 4*N*N unpadded
 * conserved; lam: N*N.  Each face is evaluated once; the reference evaluates
 * it twice (once per side) with identical inputs, hence identical bits.
 *                                               fv_up7_ducros_2d.cu:370-507 */
void OSFX(orc_up_rhs)(const REAL *Q, REAL *RHS, REAL *lam, int N, int g,
                      int order, REAL h)
{
    static const int cx[4] = { 0, 1, 2, 3 }, cy[4] = { 0, 2, 1, 3 };
    /* order + 100 rs selects the solver on the reconstructed states:
     * rs 0 HLLC (fv_up7), 1 HLL, 2 Roe (carb_fv_2d.cu:116-211) */
    const int rs = order / 100;
    order %= 100;
    int Np = N + 2 * g;
    size_t Np2 = (size_t)Np * Np, N2 = (size_t)N * N;
    REAL *Fx = (REAL *)malloc(sizeof(REAL) * 4 * (size_t)(N + 1) * N);
    REAL *Fy = (REAL *)malloc(sizeof(REAL) * 4 * (size_t)(N + 1) * N);
    for (int j = 0; j < N; j++)
        for (int i = 0; i <= N; i++) {       /* x-face i-1/2 of row j */
            ptrdiff_t b = (ptrdiff_t)(j + g) * Np + (i + g);
            REAL F[4];
            OSFX(face)(Q, Np2, b, 1, order, rs, cx, F);
            for (int q = 0; q < 4; q++) Fx[((size_t)q * N + j) * (N + 1) + i] = F[q];
        }
    for (int j = 0; j <= N; j++)             /* y-face j-1/2 of column i */
        for (int i = 0; i < N; i++) {
            ptrdiff_t b = (ptrdiff_t)(j + g) * Np + (i + g);
            REAL F[4];
            OSFX(face)(Q, Np2, b, Np, order, rs, cy, F);
            for (int q = 0; q < 4; q++) Fy[((size_t)q * (N + 1) + j) * N + i] = F[q];
        }
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            size_t k = (size_t)j * N + i;
            for (int q = 0; q < 4; q++) {
                REAL fm = Fx[((size_t)q * N + j) * (N + 1) + i];
                REAL fp = Fx[((size_t)q * N + j) * (N + 1) + i + 1];
                REAL gm = Fy[((size_t)q * (N + 1) + j) * N + i];
                REAL gp = Fy[((size_t)q * (N + 1) + j + 1) * N + i];
                RHS[q * N2 + k] = -(fp - fm) / h - (gp - gm) / h;
            }
            size_t c = (size_t)(j + g) * Np + (i + g);
            REAL r0 = Q[c], u0 = Q[Np2 + c], v0 = Q[2 * Np2 + c], p0 = Q[3 * Np2 + c];
            lam[k] = OFABS(u0) + OFABS(v0) + OSFX(snd)(p0, r0);
        }
    free(Fx);
    free(Fy);
}

/* Ghost-ring fill of a padded primitive state.
 *   bc 0: reflecting walls, u flipped in x-ghosts, v in y-ghosts
 *                                               fv_up7_ducros_2d.cu:338-362
 *   bc 1: periodic                              keep_fv_euler_2d.cu:224-243
 *   bc 2: transmissive (zero-gradient copy of the nearest interior cell, the
 *         right-boundary rule of carb_fv_2d.cu:245-247 applied on every side) */
void OSFX(orc_bc)(REAL *Q, int N, int g, int bc)
{
    int Np = N + 2 * g;
    size_t Np2 = (size_t)Np * Np;
    for (int jp = 0; jp < Np; jp++)
        for (int ip = 0; ip < Np; ip++) {
            int gx = (ip < g || ip >= N + g), gy = (jp < g || jp >= N + g);
            if (!gx && !gy) continue;
            int ir = ip, jr = jp;
            if (bc == 0) {
                if (ip < g) ir = 2 * g - 1 - ip; else if (ip >= N + g) ir = 2 * (N + g) - 1 - ip;
                if (jp < g) jr = 2 * g - 1 - jp; else if (jp >= N + g) jr = 2 * (N + g) - 1 - jp;
            } else if (bc == 1) {
                if (ip < g) ir = ip + N; else if (ip >= N + g) ir = ip - N;
                if (jp < g) jr = jp + N; else if (jp >= N + g) jr = jp - N;
            } else {
                if (ip < g) ir = g; else if (ip >= N + g) ir = N + g - 1;
                if (jp < g) jr = g; else if (jp >= N + g) jr = N + g - 1;
            }
            for (int q = 0; q < 4; q++) {
                REAL v = Q[q * Np2 + (size_t)jr * Np + ir];
                if (bc == 0 && q == 1 && gx) v = -v;
                if (bc == 0 && q == 2 && gy) v = -v;
                Q[q * Np2 + (size_t)jp * Np + ip] = v;
            }
        }
}

/* One SSP-RK3 stage on the interior, primitives in and out, conserved
 * combination, floors rho,p >= 1e-14 afterwards.
 *   stage 1: U1 = U0 + dt L(U0)
 *   stage 2: U2 = 3/4 U0 + 1/4 (U1 + dt L(U1))
 *   stage 3: U  = 1/3 U0 + 2/3 (U2 + dt L(U2))  fv_up7_ducros_2d.cu:531-590 */
void OSFX(orc_rk3)(int stage, REAL *Uo, const REAL *U0, const REAL *Uk,
                   const REAL *Lr, REAL dt, int N, int g)
{
    int Np = N + 2 * g;
    size_t Np2 = (size_t)Np * Np, N2 = (size_t)N * N;
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            size_t k = (size_t)j * N + i, c = (size_t)(j + g) * Np + (i + g);
            REAL w0[4], wk[4], c0[4], ck[4], cv[4], wp[4];
            for (int q = 0; q < 4; q++) { w0[q] = U0[q * Np2 + c]; wk[q] = Uk[q * Np2 + c]; }
            OSFX(p2c)(w0, c0);
            OSFX(p2c)(wk, ck);
            for (int q = 0; q < 4; q++) {
                REAL l = Lr[q * N2 + k];
                if (stage == 1)      cv[q] = c0[q] + dt * l;
                else if (stage == 2) cv[q] = RL(0.75) * c0[q] + RL(0.25) * (ck[q] + dt * l);
                else                 cv[q] = (RL(1.) / RL(3.)) * c0[q] + (RL(2.) / RL(3.)) * (ck[q] + dt * l);
            }
            OSFX(c2p)(cv, wp);
            wp[0] = wp[0] > RL(1e-14) ? wp[0] : RL(1e-14);
            wp[3] = wp[3] > RL(1e-14) ? wp[3] : RL(1e-14);
            for (int q = 0; q < 4; q++) Uo[q * Np2 + c] = wp[q];
        }
}

/* max over n values starting from 0 (NaN entries are skipped by fmax)
 *                                               fv_up7_ducros_2d.cu:593-612 */
REAL OSFX(orc_max)(const REAL *x, size_t n)
{
    REAL m = RL(0.);
    for (size_t k = 0; k < n; k++) m = OFMAX(m, x[k]);
    return m;
}

/* Time loop of fv_up7_ducros_2d.cu:990-1032: dt = CFL h / lam_max, clamped
 * so that t lands on t_stop; stops after max_steps steps, at t >= t_stop, on
 * a non-positive lam_max (status 1) or on dt < 1e-14 (status 2).
 * U: padded primitive state with its ghosts filled; advanced in place.
 * info (optional): {t, steps, lam_max of the final state, last dt}.        */
int OSFX(orc_up_run)(REAL *U, int N, int g, int order, int bc, REAL h, REAL cfl,
                     int max_steps, double t_stop, double info[4])
{
    int Np = N + 2 * g;
    size_t nP = (size_t)4 * Np * Np, n1 = (size_t)N * N;
    REAL *U0 = (REAL *)malloc(sizeof(REAL) * nP), *U1 = (REAL *)malloc(sizeof(REAL) * nP);
    REAL *U2 = (REAL *)malloc(sizeof(REAL) * nP), *L = (REAL *)malloc(sizeof(REAL) * 4 * n1);
    REAL *lam = (REAL *)malloc(sizeof(REAL) * n1);
    memcpy(U1, U, sizeof(REAL) * nP);
    memcpy(U2, U, sizeof(REAL) * nP);
    OSFX(orc_up_rhs)(U, L, lam, N, g, order, h);
    REAL lmax = OSFX(orc_max)(lam, n1);
    REAL t = RL(0.), dt = RL(0.), ts = (REAL)t_stop;
    int step = 0, status = 0;
    while (step < max_steps && t < ts) {
        if (!(lmax > RL(0.))) { status = 1; break; }
        dt = cfl * h / lmax;
        if (t + dt > ts) dt = ts - t;
        if (dt < RL(1e-14)) { status = 2; break; }
        memcpy(U0, U, sizeof(REAL) * nP);
        OSFX(orc_rk3)(1, U1, U0, U0, L, dt, N, g);
        OSFX(orc_bc)(U1, N, g, bc);
        OSFX(orc_up_rhs)(U1, L, lam, N, g, order, h);
        OSFX(orc_rk3)(2, U2, U0, U1, L, dt, N, g);
        OSFX(orc_bc)(U2, N, g, bc);
        OSFX(orc_up_rhs)(U2, L, lam, N, g, order, h);
        OSFX(orc_rk3)(3, U, U0, U2, L, dt, N, g);
        OSFX(orc_bc)(U, N, g, bc);
        OSFX(orc_up_rhs)(U, L, lam, N, g, order, h);
        lmax = OSFX(orc_max)(lam, n1);
        t += dt;
        step++;
    }
    if (info) { info[0] = (double)t; info[1] = step; info[2] = (double)lmax; info[3] = (double)dt; }
    free(U0); free(U1); free(U2); free(L); free(lam);
    return status;
}

/* Circular Sod initial state (primitives, interior only), tanh-smoothed
 * over one cell: rho 0.125 -> 11, p 0.1 -> 10 inside r < 0.25
 *                                               fv_up7_ducros_2d.cu:618-639 */
void OSFX(orc_ic_sod)(REAL *U, int N, int g, REAL h)
{
    int Np = N + 2 * g;
    size_t Np2 = (size_t)Np * Np;
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            REAL xc = ((REAL)i + RL(0.5)) * h, yc = ((REAL)j + RL(0.5)) * h;
            REAL r = OSQRT((xc - RL(0.5)) * (xc - RL(0.5)) + (yc - RL(0.5)) * (yc - RL(0.5)));
            REAL delta = RL(1.0) * h;
            REAL phi = RL(0.5) * (RL(1.) + OTANH((RL(0.25) - r) / delta));
            size_t c = (size_t)(j + g) * Np + (i + g);
            U[c] = RL(0.125) + RL(10.875) * phi;
            U[Np2 + c] = RL(0.);
            U[2 * Np2 + c] = RL(0.);
            U[3 * Np2 + c] = RL(0.1) + RL(9.9) * phi;
        }
}
