/*
 * fvb_oracle_keep.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * CPU restatement of the KEEP path of fvStuff's keep_fv_euler_2d.cu:
 * collocated FV on conserved cell averages, ECKEP entropy-conserving /
 * kinetic-energy-preserving central flux, JST 4th-order background
 * dissipation in smooth regions and MOVERS-RH scalar dissipation where the
 * entropy-distance sensor fires, SSP-RK3, periodic ghosts (g = 2).  FP64.
 * Association order follows the reference so the host build of the
 * reference's kernels gives the same bits (tests/test_oracle_pin.py).
 *
 * Layout: padded SoA of conserved variables [rho, rho u, rho v, E],
 * Q[q*Np*Np + jp*Np + ip], Np = N + 4        -- keep_fv_euler_2d.cu:60-80
 */

#define KG 1.4                     /* gamma              keep_fv:47 */
#define K_DELTA 1e-16              /* alpha_3 floor      keep_fv:52 */
#define K_THETA 0.1                /* sonic fix Theta    keep_fv:53 */
#define K_HESQ 12.0                /* sensor scaling q   keep_fv:56 */
#define K_HESEPS 0.05              /* sensor threshold   keep_fv:57 */
#define K_JST (1.0 / 32.0)         /* JST coefficient    keep_fv:58 */

/* c = sqrt(gamma p / rho), no clamp              keep_fv_euler_2d.cu:85-89 */
static inline double k_snd(double rho, double p) { return sqrt(KG * p / rho); }

/*                                                keep_fv_euler_2d.cu:91-96 */
static inline double k_pres(double rho, double mx, double my, double E)
{
    double u = mx / rho, v = my / rho;
    return (KG - 1.) * (E - 0.5 * rho * (u * u + v * v));
}

/* primitives with floors rho, p >= 1e-14        keep_fv_euler_2d.cu:99-110 */
static inline void k_prim(const double *Q, size_t Np2, size_t c, double W[4])
{
    double rho = fmax(Q[c], 1e-14), mx = Q[Np2 + c], my = Q[2 * Np2 + c], E = Q[3 * Np2 + c];
    W[0] = rho;
    W[1] = mx / rho;
    W[2] = my / rho;
    W[3] = fmax(k_pres(rho, mx, my, E), 1e-14);
}

/* conserved with the density floor             keep_fv_euler_2d.cu:113-120 */
static inline void k_cons(const double *Q, size_t Np2, size_t c, double U[4])
{
    U[0] = fmax(Q[c], 1e-14);
    U[1] = Q[Np2 + c];
    U[2] = Q[2 * Np2 + c];
    U[3] = Q[3 * Np2 + c];
}

/* entropy variables, s = ln(p / rho^gamma)     keep_fv_euler_2d.cu:123-132 */
static inline void k_evars(const double W[4], double V[4])
{
    double rho = W[0], u = W[1], v = W[2], p = W[3];
    double s = log(p / pow(rho, KG));
    V[0] = (KG - s) / (KG - 1.) - rho * (u * u + v * v) / (2. * p);
    V[1] = rho * u / p;
    V[2] = rho * v / p;
    V[3] = -rho / p;
}

/* ECKEP central flux (Cartesian) and the MOVERS-RH coefficient alpha_S
 *                                               keep_fv_euler_2d.cu:145-219 */
static void k_flux(const double WL[4], const double WR[4], double nx, double ny,
                   double Fec[4], double *alphaS)
{
    double rL = WL[0], uL = WL[1], vL = WL[2], pL = WL[3];
    double rR = WR[0], uR = WR[1], vR = WR[2], pR = WR[3];
    double unL = uL * nx + vL * ny, utL = -uL * ny + vL * nx;
    double unR = uR * nx + vR * ny, utR = -uR * ny + vR * nx;
    double EL = pL / (KG - 1.) + 0.5 * rL * (unL * unL + utL * utL);
    double ER = pR / (KG - 1.) + 0.5 * rR * (unR * unR + utR * utR);
    double UL[4] = { rL, rL * unL, rL * utL, EL };
    double UR[4] = { rR, rR * unR, rR * utR, ER };
    double FL[4] = { rL * unL, rL * unL * unL + pL, rL * unL * utL, (EL + pL) * unL };
    double FR[4] = { rR * unR, rR * unR * unR + pR, rR * unR * utR, (ER + pR) * unR };
    double sL = log(pL / pow(rL, KG)), sR = log(pR / pow(rR, KG));
    double VL[4] = { (KG - sL) / (KG - 1.) - rL * (unL * unL + utL * utL) / (2. * pL),
                     rL * unL / pL, rL * utL / pL, -rL / pL };
    double VR[4] = { (KG - sR) / (KG - 1.) - rR * (unR * unR + utR * utR) / (2. * pR),
                     rR * unR / pR, rR * utR / pR, -rR / pR };
    double dV[4] = { VR[0] - VL[0], VR[1] - VL[1], VR[2] - VL[2], VR[3] - VL[3] };
    double dpsi = rR * unR - rL * unL;

    double Fc0 = 0.5 * (FL[0] + FR[0]);
    double unb = 0.5 * (unL + unR), utb = 0.5 * (utL + utR), pb = 0.5 * (pL + pR);
    double Fc1 = Fc0 * unb + pb;
    double Fc2 = Fc0 * utb;
    double Feb = 0.5 * (FL[3] + FR[3]);
    double num = dV[0] * Fc0 + dV[1] * Fc1 + dV[2] * Fc2 + dV[3] * Feb - dpsi;
    double Fc3 = Feb - (num / (dV[3] * dV[3] + K_DELTA)) * dV[3];
    Fec[0] = Fc0;
    Fec[1] = Fc1 * nx - Fc2 * ny;
    Fec[2] = Fc1 * ny + Fc2 * nx;
    Fec[3] = Fc3;

    double rav = 0.5 * (rL + rR);
    double aav = k_snd(fmax(rav, 1e-14), fmax(pb, 1e-14));
    double l1 = fabs(unb - aav), l2 = fabs(unb), l3 = fabs(unb + aav);
    double lmin = fmin(l1, fmin(l2, l3)), lmax = fmax(l1, fmax(l2, l3));
    double aS = lmax;
    for (int q = 0; q < 4; q++) {
        double dU = UR[q] - UL[q], sk;
        if (fabs(dU) < 1e-12) {
            sk = lmin;
        } else {
            sk = fabs((FR[q] - FL[q]) / dU);
            if (sk >= lmax) sk = lmax;
            else if (sk <= lmin) sk = lmin;
        }
        if (sk < aS) aS = sk;
    }
    if (aS < K_THETA) aS = (aS * aS + K_THETA * K_THETA) / (2. * K_THETA);
    *alphaS = aS;
}

/* |(U_n - U_c) . (V_n - V_c)|                   keep_fv_euler_2d.cu:249-258 */
static double k_edist(const double Wc[4], const double Uc[4], const double Wn[4], const double Un[4])
{
    double Vc[4], Vn[4], ed = 0.;
    k_evars(Wc, Vc);
    k_evars(Wn, Vn);
    for (int q = 0; q < 4; q++) ed += (Un[q] - Uc[q]) * (Vn[q] - Vc[q]);
    return fabs(ed);
}

/* phi = 1 where 1 - exp(-q ed/ed_max) > eps    keep_fv_euler_2d.cu:280-286 */
static double k_phi(double ed, double edmax)
{
    double sed = ed / (edmax + 1e-30);
    double phi = 1. - exp(-K_HESQ * sed);
    return (phi > K_HESEPS) ? 1. : 0.;
}

/* per-cell entropy distance, max over the right and top faces
 *                                               keep_fv_euler_2d.cu:260-277 */
void orc_keep_ed(const double *Q, double *ed, int N)
{
    int g = 2, Np = N + 2 * g;
    size_t Np2 = (size_t)Np * Np;
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            size_t c = (size_t)(j + g) * Np + (i + g);
            double Wc[4], Uc[4], Wx[4], Ux[4], Wy[4], Uy[4];
            k_prim(Q, Np2, c, Wc); k_cons(Q, Np2, c, Uc);
            k_prim(Q, Np2, c + 1, Wx); k_cons(Q, Np2, c + 1, Ux);
            k_prim(Q, Np2, c + Np, Wy); k_cons(Q, Np2, c + Np, Uy);
            ed[(size_t)j * N + i] = fmax(k_edist(Wc, Uc, Wx, Ux), k_edist(Wc, Uc, Wy, Uy));
        }
}

/* flux through the face between padded cells a (left/bottom) and b = a + st,
 * F = F_EC + (1-phi) JST + phi RH               keep_fv_euler_2d.cu:330-345 */
static void k_face(const double *Q, size_t Np2, size_t a, size_t st, double nx, double ny,
                   double edmax, double F[4])
{
    double WL[4], WR[4], UL[4], UR[4], Up2[4], Um1[4], fec[4], aS;
    k_prim(Q, Np2, a, WL); k_prim(Q, Np2, a + st, WR);
    k_cons(Q, Np2, a, UL); k_cons(Q, Np2, a + st, UR);
    k_cons(Q, Np2, a + 2 * st, Up2); k_cons(Q, Np2, a - st, Um1);
    k_flux(WL, WR, nx, ny, fec, &aS);
    double unL = WL[1] * nx + WL[2] * ny, unR = WR[1] * nx + WR[2] * ny;
    double aR = k_snd(0.5 * (WL[0] + WR[0]), 0.5 * (WL[3] + WR[3]));
    double lamt = fmax(fabs(unL), fabs(unR)) + aR;
    double aJST = K_JST * lamt;
    double phi = k_phi(k_edist(WL, UL, WR, UR), edmax);
    for (int q = 0; q < 4; q++) {
        double jst = aJST * (Up2[q] - 3. * UR[q] + 3. * UL[q] - Um1[q]);
        double rh = -0.5 * aS * (UR[q] - UL[q]);
        F[q] = fec[q] + (1. - phi) * jst + phi * rh;
    }
}

/* residual of the conserved variables and lam = (|u|+c) + (|v|+c); each face
 * once (the reference evaluates it from both sides with the same inputs)
 *                                               keep_fv_euler_2d.cu:298-369 */
void orc_keep_rhs(const double *Q, double *RHS, double *lam, int N, double h, double edmax)
{
    int g = 2, Np = N + 2 * g;
    size_t Np2 = (size_t)Np * Np, N2 = (size_t)N * N;
    double *Fx = (double *)malloc(sizeof(double) * 4 * (size_t)(N + 1) * N);
    double *Fy = (double *)malloc(sizeof(double) * 4 * (size_t)(N + 1) * N);
    for (int j = 0; j < N; j++)
        for (int i = 0; i <= N; i++) {
            double F[4];
            k_face(Q, Np2, (size_t)(j + g) * Np + (i + g - 1), 1, 1., 0., edmax, F);
            for (int q = 0; q < 4; q++) Fx[((size_t)q * N + j) * (N + 1) + i] = F[q];
        }
    for (int j = 0; j <= N; j++)
        for (int i = 0; i < N; i++) {
            double F[4];
            k_face(Q, Np2, (size_t)(j + g - 1) * Np + (i + g), (size_t)Np, 0., 1., edmax, F);
            for (int q = 0; q < 4; q++) Fy[((size_t)q * (N + 1) + j) * N + i] = F[q];
        }
    double inv_h = 1. / h;
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            size_t k = (size_t)j * N + i;
            for (int q = 0; q < 4; q++) {
                double fr = Fx[((size_t)q * N + j) * (N + 1) + i + 1];
                double fl = Fx[((size_t)q * N + j) * (N + 1) + i];
                double ft = Fy[((size_t)q * (N + 1) + j + 1) * N + i];
                double fb = Fy[((size_t)q * (N + 1) + j) * N + i];
                RHS[q * N2 + k] = -(fr - fl + ft - fb) * inv_h;
            }
            double W[4];
            k_prim(Q, Np2, (size_t)(j + g) * Np + (i + g), W);
            double cs = k_snd(W[0], W[3]);
            lam[k] = (fabs(W[1]) + cs) + (fabs(W[2]) + cs);
        }
    free(Fx);
    free(Fy);
}

/* Uo = ca Ua + cb Ub + cl dt L, floors rho, E >= 1e-14
 *                                               keep_fv_euler_2d.cu:374-393 */
void orc_keep_rk(double *Uo, const double *Ua, const double *Ub, const double *L,
                 double ca, double cb, double cl, double dt, int N)
{
    int g = 2, Np = N + 2 * g;
    size_t Np2 = (size_t)Np * Np, N2 = (size_t)N * N;
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            size_t k = (size_t)j * N + i, c = (size_t)(j + g) * Np + (i + g);
            for (int q = 0; q < 4; q++)
                Uo[q * Np2 + c] = ca * Ua[q * Np2 + c] + cb * Ub[q * Np2 + c] + cl * dt * L[q * N2 + k];
            Uo[c] = fmax(Uo[c], 1e-14);
            Uo[3 * Np2 + c] = fmax(Uo[3 * Np2 + c], 1e-14);
        }
}

/* residual with the sensor normalised by the global entropy-distance max
 *                                               keep_fv_euler_2d.cu:640-645 */
static void k_rhs_of(const double *U, double *L, double *lam, double *ed, int N, double h)
{
    orc_keep_ed(U, ed, N);
    double edmax = orc_max_f64(ed, (size_t)N * N);
    orc_keep_rhs(U, L, lam, N, h, edmax);
}

/* time loop of keep_fv_euler_2d.cu:691-725 (same dt rule as the UP7 path) */
int orc_keep_run(double *U, int N, double h, double cfl, int max_steps, double t_stop,
                 double info[4])
{
    int g = 2, Np = N + 2 * g;
    size_t nP = (size_t)4 * Np * Np, n1 = (size_t)N * N;
    double *U0 = (double *)malloc(sizeof(double) * nP), *U1 = (double *)malloc(sizeof(double) * nP);
    double *U2 = (double *)malloc(sizeof(double) * nP), *L = (double *)malloc(sizeof(double) * 4 * n1);
    double *lam = (double *)malloc(sizeof(double) * n1), *ed = (double *)malloc(sizeof(double) * n1);
    memcpy(U1, U, sizeof(double) * nP);
    memcpy(U2, U, sizeof(double) * nP);
    k_rhs_of(U, L, lam, ed, N, h);
    double lmax = orc_max_f64(lam, n1), t = 0., dt = 0.;
    int step = 0, status = 0;
    while (step < max_steps && t < t_stop) {
        if (!(lmax > 0.)) { status = 1; break; }
        dt = cfl * h / lmax;
        if (t + dt > t_stop) dt = t_stop - t;
        if (dt < 1e-14) { status = 2; break; }
        memcpy(U0, U, sizeof(double) * nP);
        orc_keep_rk(U1, U0, U0, L, 1., 0., 1., dt, N);
        orc_bc_f64(U1, N, g, 1);
        k_rhs_of(U1, L, lam, ed, N, h);
        orc_keep_rk(U2, U0, U1, L, 0.75, 0.25, 0.25, dt, N);
        orc_bc_f64(U2, N, g, 1);
        k_rhs_of(U2, L, lam, ed, N, h);
        orc_keep_rk(U, U0, U2, L, 1. / 3., 2. / 3., 2. / 3., dt, N);
        orc_bc_f64(U, N, g, 1);
        k_rhs_of(U, L, lam, ed, N, h);
        lmax = orc_max_f64(lam, n1);
        t += dt;
        step++;
    }
    if (info) { info[0] = t; info[1] = step; info[2] = lmax; info[3] = dt; }
    free(U0); free(U1); free(U2); free(L); free(lam); free(ed);
    return status;
}

/* circular Sod in conserved variables, rho 0.125 -> 1, p 0.1 -> 1
 *                                               keep_fv_euler_2d.cu:448-469 */
void orc_keep_ic_sod(double *Q, int N, double h)
{
    int g = 2, Np = N + 2 * g;
    size_t Np2 = (size_t)Np * Np;
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            double xc = (i + 0.5) * h, yc = (j + 0.5) * h;
            double r = sqrt((xc - 0.5) * (xc - 0.5) + (yc - 0.5) * (yc - 0.5));
            double delta = 1.0 * h;
            double phi = 0.5 * (1. + tanh((0.25 - r) / delta));
            double rho = 0.125 + (1.0 - 0.125) * phi;
            double p = 0.1 + (1.0 - 0.1) * phi;
            size_t c = (size_t)(j + g) * Np + (i + g);
            Q[c] = rho; Q[Np2 + c] = 0.; Q[2 * Np2 + c] = 0.; Q[3 * Np2 + c] = p / (KG - 1.);
        }
}

/* stationary low-Mach vortex with Mach number eps
 *                                               keep_fv_euler_2d.cu:471-513 */
static void k_lmv_exact(double x, double y, double p0, double *rho, double *u, double *v, double *p)
{
    double dx = x - 0.5, dy = y - 0.5, r = sqrt(dx * dx + dy * dy);
    double vp = (r < 0.2) ? 5. * r : (r < 0.4) ? 2. - 5. * r : 0.;
    double ir = (r > 1e-30) ? 1. / r : 0.;
    *rho = 1.;
    *u = -vp * dy * ir;
    *v = vp * dx * ir;
    if (r < 0.2) *p = p0 + 12.5 * r * r;
    else if (r < 0.4) *p = p0 + 4. * log(5. * r) + 4. - 20. * r + 12.5 * r * r;
    else *p = p0 + 4. * log(2.) - 2.;
}

void orc_keep_ic_lmv(double *Q, int N, double h, double eps)
{
    const double p0 = 1. / (KG * eps * eps) - 0.5;
    int g = 2, Np = N + 2 * g;
    size_t Np2 = (size_t)Np * Np;
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            double rho, u, v, p;
            k_lmv_exact((i + 0.5) * h, (j + 0.5) * h, p0, &rho, &u, &v, &p);
            size_t c = (size_t)(j + g) * Np + (i + g);
            Q[c] = rho; Q[Np2 + c] = rho * u; Q[2 * Np2 + c] = rho * v;
            Q[3 * Np2 + c] = p / (KG - 1.) + 0.5 * rho * (u * u + v * v);
        }
}

/* L2 errors of rho and p against the exact stationary vortex
 *                                               keep_fv_euler_2d.cu:516-536 */
void orc_keep_err_lmv(const double *Q, int N, double h, double eps, double out[2])
{
    const double p0 = 1. / (KG * eps * eps) - 0.5;
    int g = 2, Np = N + 2 * g;
    size_t Np2 = (size_t)Np * Np;
    double sr = 0., sp = 0.;
    for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++) {
            double re, ue, ve, pe;
            k_lmv_exact((i + 0.5) * h, (j + 0.5) * h, p0, &re, &ue, &ve, &pe);
            size_t c = (size_t)(j + g) * Np + (i + g);
            double rho = fmax(Q[c], 1e-14);
            double p = k_pres(rho, Q[Np2 + c], Q[2 * Np2 + c], Q[3 * Np2 + c]);
            double dr = rho - re, dp = p - pe;
            sr += dr * dr * h * h;
            sp += dp * dp * h * h;
        }
    out[0] = sqrt(sr);
    out[1] = sqrt(sp);
}
