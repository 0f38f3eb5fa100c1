/*
 * fvb_oracle_d2av.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * CPU restatement of the scheme kept in fvStuff's fv_up7_ducros_2d.cu.bak
 * (the earlier form of fv_up7), FP64: UP-order reconstruction of the
 * conserved variables, HLLC on the reconstructed states, and a D2
 * artificial viscosity whose Ducros weight S_D comes from the 6th-order
 * velocity divergence; SSP-RK3 on conserved variables without floors.
 *
 * The reference reads an unpadded N x N array through a reflecting fetch
 * (fv_up7_ducros_2d.cu.bak:49-62).  Here the state is padded with
 * g = max((order + 1) / 2, 3) ghost layers filled by orc_bc_f64 (bc 0
 * reflects exactly as that fetch does; bc 1 periodic and bc 2 transmissive
 * are the other two ghost rules of this library), and every offset the
 * scheme reads (+-g along a row or a column) lands in that ring.
 *
 * Operations keep the reference's association order, so compiled without
 * FMA contraction this is bit-identical to the reference's own kernels
 * built for the host (tests/test_oracle_pin.py).  upface_f64 and orc_bc_f64
 * come from fvb_oracle_up7.h, whose UP3/5/7/9 expressions are the .bak's.
 *
 * Layout: padded SoA of conserved variables (rho, rho u, rho v, E),
 * Q[q*Np*Np + jp*Np + ip], Np = N + 2g.
 */

#define D2_GAM 1.4

static inline int d2_ghost(int order)
{
    int g = (order + 1) / 2;
    return g > 3 ? g : 3;
}

/* conserved -> p, c, u, v (no density floor; c^2 floored at 1e-14)
 *                                         fv_up7_ducros_2d.cu.bak:65-74 */
static inline void d2_prim(double rho, double mx, double my, double E,
                           double *p, double *c, double *u, double *v)
{
    *u = mx / rho;
    *v = my / rho;
    *p = (D2_GAM - 1.0) * (E - 0.5 * (mx * (*u) + my * (*v)));
    double cs2 = D2_GAM * (*p) / rho;
    *c = sqrt(cs2 > 1e-14 ? cs2 : 1e-14);
}

/* HLLC of conserved face states in the face-normal frame: U = (rho, m_n,
 * m_t, E), F = (mass, normal mom., tangential mom., energy).  The x-face
 * solver is this with (m_n, m_t) = (rho u, rho v); the y-face solver is the
 * same arithmetic with the two momenta swapped in and out (the swap leaves
 * every operation's operands unchanged; IEEE addition commutes).
 *                                         fv_up7_ducros_2d.cu.bak:202-282 */
static void d2_hllc(const double UL[4], const double UR[4], double F[4])
{
    double pL, cL, uL, vL, pR, cR, uR, vR;
    d2_prim(UL[0], UL[1], UL[2], UL[3], &pL, &cL, &uL, &vL);
    d2_prim(UR[0], UR[1], UR[2], UR[3], &pR, &cR, &uR, &vR);
    double SL = fmin(uL - cL, uR - cR);
    double SR = fmax(uL + cL, uR + cR);
    if (SL >= 0.0) {
        F[0] = UL[1]; F[1] = UL[1] * uL + pL; F[2] = UL[1] * vL; F[3] = (UL[3] + pL) * uL;
        return;
    }
    if (SR <= 0.0) {
        F[0] = UR[1]; F[1] = UR[1] * uR + pR; F[2] = UR[1] * vR; F[3] = (UR[3] + pR) * uR;
        return;
    }
    double dL = UL[0] * (SL - uL), dR = UR[0] * (SR - uR);
    double Ss = (pR - pL + dL * uL - dR * uR) / (dL - dR);
    int left = Ss >= 0.0;
    const double *UK = left ? UL : UR;
    double pK = left ? pL : pR, uK = left ? uL : uR, vK = left ? vL : vR, SK = left ? SL : SR;
    double fact = UK[0] * (SK - uK) / (SK - Ss);
    double Us[4];
    Us[0] = fact;
    Us[1] = fact * Ss;
    Us[2] = fact * vK;
    Us[3] = fact * (UK[3] / UK[0] + (Ss - uK) * (Ss + pK / (UK[0] * (SK - uK))));
    double FK[4] = { UK[1], UK[1] * uK + pK, UK[1] * vK, (UK[3] + pK) * uK };
    for (int q = 0; q < 4; q++) F[q] = FK[q] + SK * (Us[q] - UK[q]);
}

/* flux through the face whose right/top cell is padded index b; st = 1 for
 * an x-face, Np for a y-face; the stencil is cells b - h .. b + h - 1
 * (h = (order + 1) / 2)                    fv_up7_ducros_2d.cu.bak:300-337 */
static void d2_face(const double *Q, size_t Np2, ptrdiff_t b, ptrdiff_t st, int order, int yface,
                    double F[4])
{
    int hw = (order + 1) / 2, sw = 2 * hw;
    double s[10], L[4], R[4], UL[4], UR[4], Fn[4];
    for (int q = 0; q < 4; q++) {
        for (int d = 0; d < sw; d++) s[d] = Q[q * Np2 + b + (ptrdiff_t)(d - hw) * st];
        upface_f64(order, s, &L[q], &R[q]);
    }
    int qn = yface ? 2 : 1, qt = yface ? 1 : 2;
    UL[0] = L[0]; UL[1] = L[qn]; UL[2] = L[qt]; UL[3] = L[3];
    UR[0] = R[0]; UR[1] = R[qn]; UR[2] = R[qt]; UR[3] = R[3];
    d2_hllc(UL, UR, Fn);
    F[0] = Fn[0]; F[qn] = Fn[1]; F[qt] = Fn[2]; F[3] = Fn[3];
}

/* velocity with the density floored at 1e-14 (the sensor's form)
 *                                         fv_up7_ducros_2d.cu.bak:347-351 */
static inline double d2_vel(const double *Q, size_t Np2, size_t e, int q)
{
    double r = Q[e];
    r = r > 1e-14 ? r : 1e-14;
    return Q[q * Np2 + e] / r;
}

/* Ducros weight S_D of cell e from the 6th-order divergence, compressions
 * only                                     fv_up7_ducros_2d.cu.bak:344-357 */
static double d2_sensor(const double *Q, size_t Np2, size_t e, int Np, double h, double sc, double c0)
{
    static const double wc[6] = { -1., 9., -45., 45., -9., 1. };
    static const int wo[6] = { -3, -2, -1, 1, 2, 3 };
    double du_dx = 0., dv_dy = 0.;
    for (int m = 0; m < 6; m++) {
        du_dx += wc[m] * d2_vel(Q, Np2, e + wo[m], 1);
        dv_dy += wc[m] * d2_vel(Q, Np2, e + (ptrdiff_t)wo[m] * Np, 2);
    }
    du_dx /= 60. * h;
    dv_dy /= 60. * h;
    double div_u = du_dx + dv_dy;
    if (div_u > 0.) div_u = 0.;
    double sos2 = (sc / (h * h)) * c0 * c0;
    return (div_u * div_u) / (div_u * div_u + sos2 + 1e-40);
}

/* |u| + c and |v| + c of cell e             fv_up7_ducros_2d.cu.bak:86-98 */
static inline void d2_lamxy(const double *Q, size_t Np2, size_t e, double *lx, double *ly)
{
    double p, c, u, v;
    d2_prim(Q[e], Q[Np2 + e], Q[2 * Np2 + e], Q[3 * Np2 + e], &p, &c, &u, &v);
    *lx = fabs(u) + c;
    *ly = fabs(v) + c;
}

/* residual of the conserved variables (4 x N x N, unpadded) and per-cell
 * lam = |u| + |v| + c (N x N) of a padded conserved state Q with ghosts
 * filled; C2, Cg: Ducros-gated and global D2 coefficients, sc: sensor
 * sound-speed scale                        fv_up7_ducros_2d.cu.bak:287-390 */
void orc_d2av_rhs(const double *Q, double *RHS, double *lam, int N, int order, double h,
                  double C2, double Cg, double sc)
{
    int g = d2_ghost(order), Np = N + 2 * g;
    size_t Np2 = (size_t)Np * Np, N2 = (size_t)N * N;
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            size_t e = (size_t)(j + g) * Np + (i + g);
            double Fm[4], Fp[4], Gm[4], Gp[4];
            d2_face(Q, Np2, (ptrdiff_t)e, 1, order, 0, Fm);
            d2_face(Q, Np2, (ptrdiff_t)e + 1, 1, order, 0, Fp);
            d2_face(Q, Np2, (ptrdiff_t)e, Np, order, 1, Gm);
            d2_face(Q, Np2, (ptrdiff_t)e + Np, Np, order, 1, Gp);
            double p0, c0, u0, v0;
            d2_prim(Q[e], Q[Np2 + e], Q[2 * Np2 + e], Q[3 * Np2 + e], &p0, &c0, &u0, &v0);
            double S_D = d2_sensor(Q, Np2, e, Np, h, sc, c0);
            double lam_c = fabs(u0) + fabs(v0) + c0;
            double lamx_c = fabs(u0) + c0, lamy_c = fabs(v0) + c0, lx, ly;
            d2_lamxy(Q, Np2, e + 1, &lx, &ly);
            double lhxp = 0.5 * (lamx_c + lx);
            d2_lamxy(Q, Np2, e - 1, &lx, &ly);
            double lhxm = 0.5 * (lamx_c + lx);
            d2_lamxy(Q, Np2, e + Np, &lx, &ly);
            double lhyp = 0.5 * (lamy_c + ly);
            d2_lamxy(Q, Np2, e - Np, &lx, &ly);
            double lhym = 0.5 * (lamy_c + ly);
            for (int q = 0; q < 4; q++) {
                const double *v = Q + q * Np2;
                double Uc = v[e];
                double dxp = v[e + 1] - Uc, dxm = Uc - v[e - 1];
                double dyp = v[e + Np] - Uc, dym = Uc - v[e - Np];
                double d2_duc = (C2 / h) * (lhxp * S_D * dxp - lhxm * S_D * dxm
                                            + lhyp * S_D * dyp - lhym * S_D * dym);
                double d2_glb = (Cg / h) * (lhxp * (1. - S_D) * dxp - lhxm * (1. - S_D) * dxm
                                            + lhyp * (1. - S_D) * dyp - lhym * (1. - S_D) * dym);
                double D2 = d2_duc + d2_glb;
                RHS[q * N2 + (size_t)j * N + i] = -(Fp[q] - Fm[q]) / h - (Gp[q] - Gm[q]) / h + D2;
            }
            lam[(size_t)j * N + i] = lam_c;
        }
}

/* Ducros weight of every cell (the frame panel)   fv_up7_ducros_2d.cu.bak:393-428 */
void orc_d2av_sensor(const double *Q, double *SD, int N, int order, double h, double sc)
{
    int g = d2_ghost(order), Np = N + 2 * g;
    size_t Np2 = (size_t)Np * Np;
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            size_t e = (size_t)(j + g) * Np + (i + g);
            double p0, c0, u0, v0;
            d2_prim(Q[e], Q[Np2 + e], Q[2 * Np2 + e], Q[3 * Np2 + e], &p0, &c0, &u0, &v0);
            SD[(size_t)j * N + i] = d2_sensor(Q, Np2, e, Np, h, sc, c0);
        }
}

/* SSP-RK3 stage on the interior of conserved states, no floors
 *   stage 1: U1 = U0 + dt L
 *   stage 2: U2 = 0.75 U0 + 0.25 (U1 + dt L)
 *   stage 3: U  = 1/3 U0 + 2/3 (U2 + dt L)  fv_up7_ducros_2d.cu.bak:433-446 */
void orc_d2av_rk3(int stage, double *Uo, const double *U0, const double *Uk, const double *Lr,
                  double dt, int N, int g)
{
    int Np = N + 2 * g;
    size_t Np2 = (size_t)Np * Np, N2 = (size_t)N * N;
    for (int q = 0; q < 4; q++)
        for (int j = 0; j < N; j++)
            for (int i = 0; i < N; i++) {
                size_t c = q * Np2 + (size_t)(j + g) * Np + (i + g);
                double l = Lr[q * N2 + (size_t)j * N + i];
                if (stage == 1) Uo[c] = U0[c] + dt * l;
                else if (stage == 2) Uo[c] = 0.75 * U0[c] + 0.25 * (Uk[c] + dt * l);
                else Uo[c] = (1. / 3.) * U0[c] + (2. / 3.) * (Uk[c] + dt * l);
            }
}

/* Time loop of fv_up7_ducros_2d.cu.bak:848-872 (the residual and its lam
 * at the start of each step, dt = CFL h / lam_max clamped onto t_stop, stop
 * on dt < 1e-14; status 1 also on a non-positive lam_max, which the .bak
 * would carry on through).  U: padded conserved state, ghosts filled, bc as
 * orc_bc_f64; advanced in place.  info: {t, steps, lam_max, last dt}.     */
int orc_d2av_run(double *U, int N, int order, int bc, double h, double cfl, double C2, double Cg,
                 double sc, int max_steps, double t_stop, double info[4])
{
    int g = d2_ghost(order), Np = N + 2 * g;
    size_t nP = (size_t)4 * Np * Np, n1 = (size_t)N * N;
    double *U0 = (double *)malloc(sizeof(double) * nP), *U1 = (double *)malloc(sizeof(double) * nP);
    double *U2 = (double *)malloc(sizeof(double) * nP), *L = (double *)malloc(sizeof(double) * 4 * n1);
    double *lam = (double *)malloc(sizeof(double) * n1);
    memcpy(U1, U, sizeof(double) * nP);
    memcpy(U2, U, sizeof(double) * nP);
    double t = 0., dt = 0., lmax = 0.;
    int step = 0, status = 0;
    orc_d2av_rhs(U, L, lam, N, order, h, C2, Cg, sc);
    lmax = orc_max_f64(lam, n1);
    while (step < max_steps && t < t_stop) {
        if (!(lmax > 0.)) { status = 1; break; }
        dt = cfl * h / lmax;
        if (t + dt > t_stop) dt = t_stop - t;
        if (dt < 1e-14) { status = 2; break; }
        memcpy(U0, U, sizeof(double) * nP);
        orc_d2av_rk3(1, U1, U0, U0, L, dt, N, g);
        orc_bc_f64(U1, N, g, bc);
        orc_d2av_rhs(U1, L, lam, N, order, h, C2, Cg, sc);
        orc_d2av_rk3(2, U2, U0, U1, L, dt, N, g);
        orc_bc_f64(U2, N, g, bc);
        orc_d2av_rhs(U2, L, lam, N, order, h, C2, Cg, sc);
        orc_d2av_rk3(3, U, U0, U2, L, dt, N, g);
        orc_bc_f64(U, N, g, bc);
        orc_d2av_rhs(U, L, lam, N, order, h, C2, Cg, sc);
        lmax = orc_max_f64(lam, n1);
        t += dt;
        step++;
    }
    if (info) { info[0] = t; info[1] = step; info[2] = lmax; info[3] = dt; }
    free(U0); free(U1); free(U2); free(L); free(lam);
    return status;
}

/* circular Sod of the .bak, conserved, interior only: rho 0.125 -> 10,
 * p 0.1 -> 10 inside r < 0.25, tanh-smoothed over one cell, at rest
 *                                         fv_up7_ducros_2d.cu.bak:472-491 */
void orc_d2av_ic_sod(double *U, int N, double h, int g)
{
    int Np = N + 2 * g;
    size_t Np2 = (size_t)Np * Np;
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            double xc = (i + 0.5) * h, yc = (j + 0.5) * h;
            double r = sqrt((xc - 0.5) * (xc - 0.5) + (yc - 0.5) * (yc - 0.5));
            double delta = 1.0 * h;
            double phi = 0.5 * (1. + tanh((0.25 - r) / delta));
            size_t c = (size_t)(j + g) * Np + (i + g);
            U[c] = 0.125 + 9.875 * phi;
            U[Np2 + c] = 0.;
            U[2 * Np2 + c] = 0.;
            U[3 * Np2 + c] = (0.1 + 9.9 * phi) / (D2_GAM - 1.);
        }
}
