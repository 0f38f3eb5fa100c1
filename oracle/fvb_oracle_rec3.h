/*
 * fvb_oracle_rec3.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * CPU restatement of fvStuff's fv_rec3_2d.cu in FP64 (real = reall =
 * double): unlimited 3rd-order (rec3) face reconstruction in conserved
 * variables, a pointwise Zhang-Shu scaling of each face state toward its
 * cell average, HLLC, SSP-RK3, and after every stage the a-posteriori
 * Zhang-Shu positivity limiter on non-overlapping 2x2 cell blocks.
 * Periodic, g = 2, N even.
 *
 * The reference accumulates each face flux into its two cells with
 * atomicAdd; run serially (its kernels built for the host with one thread)
 * the additions happen in cell order, which rec3_rhs reproduces literally,
 * so the restatement is bit-identical to that serial run.
 *
 * Layout: padded SoA of conserved variables (rho, rho u, rho v, E),
 * Q[q*Np*Np + jp*Np + ip], Np = N + 4.
 */

#define R3_G 2
#define R3_GAM 1.4
#define R3_PFLOOR 1e-9
#define R3_RHOFLOOR 1e-12

/* c = sqrt(gamma p / rho)                       fv_rec3_2d.cu:68-69 */
static inline double r3_snd(double rho, double p) { return sqrt(R3_GAM * p / rho); }

/* conserved point value -> floored primitives  fv_rec3_2d.cu:71-79 */
static inline void r3_w(double rho, double mx, double my, double E, double W[4])
{
    double r = fmax(rho, R3_RHOFLOOR);
    double u = mx / r, v = my / r;
    double p = (R3_GAM - 1.0) * (E - 0.5 * r * (u * u + v * v));
    W[0] = r; W[1] = u; W[2] = v; W[3] = fmax(p, R3_PFLOOR);
}

/* pressure of a conserved state                fv_rec3_2d.cu:81-87 */
static inline double r3_p(const double U[4])
{
    double r = fmax(U[0], R3_RHOFLOOR);
    double u = U[1] / r, v = U[2] / r;
    return (R3_GAM - 1.0) * (U[3] - 0.5 * r * (u * u + v * v));
}

/* HLLC with Davis bounds, each side's star state, normal frame
 * (rho, un, ut, p); the y-face relabelling of fvb_oracle_up7.h applies
 *                                              fv_rec3_2d.cu:90-123 */
static void r3_hllc(const double L[4], const double R[4], double F[4])
{
    double rL = L[0], uL = L[1], tL = L[2], pL = L[3];
    double rR = R[0], uR = R[1], tR = R[2], pR = R[3];
    double cL = r3_snd(rL, pL), cR = r3_snd(rR, pR);
    double EL = pL / (R3_GAM - 1.) + 0.5 * rL * (uL * uL + tL * tL);
    double ER = pR / (R3_GAM - 1.) + 0.5 * rR * (uR * uR + tR * tR);
    double SL = fmin(uL - cL, uR - cR), SR = fmax(uL + cL, uR + cR);
    double FL[4] = { rL * uL, rL * uL * uL + pL, rL * uL * tL, (EL + pL) * uL };
    double FR[4] = { rR * uR, rR * uR * uR + pR, rR * uR * tR, (ER + pR) * uR };
    if (SL >= 0.) { for (int q = 0; q < 4; q++) F[q] = FL[q]; return; }
    if (SR <= 0.) { for (int q = 0; q < 4; q++) F[q] = FR[q]; return; }
    double dL = rL * (SL - uL), dR = rR * (SR - uR);
    double Ss = (pR - pL + dL * uL - dR * uR) / (dL - dR);
    if (Ss >= 0.) {
        double f = rL * (SL - uL) / (SL - Ss);
        double Us[4] = { f, f * Ss, f * tL, f * (EL / rL + (Ss - uL) * (Ss + pL / (rL * (SL - uL)))) };
        double U[4] = { rL, rL * uL, rL * tL, EL };
        for (int q = 0; q < 4; q++) F[q] = FL[q] + SL * (Us[q] - U[q]);
    } else {
        double f = rR * (SR - uR) / (SR - Ss);
        double Us[4] = { f, f * Ss, f * tR, f * (ER / rR + (Ss - uR) * (Ss + pR / (rR * (SR - uR)))) };
        double U[4] = { rR, rR * uR, rR * tR, ER };
        for (int q = 0; q < 4; q++) F[q] = FR[q] + SR * (Us[q] - U[q]);
    }
}

/* Zhang-Shu scaling of a reconstructed state U toward its cell's average Ub
 * until rho and p clear their floors (linear for rho, 25-step bisection for
 * p)                                           fv_rec3_2d.cu:125-145 */
static void r3_scale(const double Ub[4], double U[4])
{
    if (U[0] < R3_RHOFLOOR) {
        double d = Ub[0] - U[0];
        double th = (d > 0.) ? (Ub[0] - R3_RHOFLOOR) / d : 0.;
        for (int q = 0; q < 4; q++) U[q] = Ub[q] + th * (U[q] - Ub[q]);
    }
    if (r3_p(U) < R3_PFLOOR) {
        double lo = 0., hi = 1.;
        for (int it = 0; it < 25; it++) {
            double mid = 0.5 * (lo + hi), V[4];
            for (int q = 0; q < 4; q++) V[q] = Ub[q] + mid * (U[q] - Ub[q]);
            if (V[0] >= R3_RHOFLOOR && r3_p(V) >= R3_PFLOOR) lo = mid; else hi = mid;
        }
        for (int q = 0; q < 4; q++) U[q] = Ub[q] + lo * (U[q] - Ub[q]);
    }
}

/* flux through the face between the cells at padded offsets b and b + st;
 * comp maps the conserved slots to the normal frame ({0,1,2,3} for x-faces,
 * {0,2,1,3} for y-faces)                       fv_rec3_2d.cu:182-243 */
static void r3_face(const double *Q, size_t Np2, ptrdiff_t b, ptrdiff_t st, const int comp[4], double F[4])
{
    double UL[4], UR[4], UbL[4], UbR[4], WL[4], WR[4], Fn[4];
    for (int q = 0; q < 4; q++) {
        const double *v = Q + (size_t)q * Np2 + b;
        double um = v[-st], uc = v[0], up = v[st], u2 = v[2 * st];
        UL[q] = (-um + 5. * uc + 2. * up) * (1. / 6.);
        UR[q] = (2. * uc + 5. * up - u2) * (1. / 6.);
        UbL[q] = uc;
        UbR[q] = up;
    }
    r3_scale(UbL, UL);
    r3_scale(UbR, UR);
    r3_w(UL[0], UL[1], UL[2], UL[3], WL);
    r3_w(UR[0], UR[1], UR[2], UR[3], WR);
    double L[4], R[4];
    for (int q = 0; q < 4; q++) { L[q] = WL[comp[q]]; R[q] = WR[comp[q]]; }
    r3_hllc(L, R, Fn);
    for (int q = 0; q < 4; q++) F[comp[q]] = Fn[q];
}

/* residual by the reference's scatter, in cell order, and the spectral
 * radius |u|+|v|+c of each cell                fv_rec3_2d.cu:166-245 */
void orc_rec3_rhs(const double *Q, double *RHS, double *lam, int N, double h)
{
    static const int cx[4] = { 0, 1, 2, 3 }, cy[4] = { 0, 2, 1, 3 };
    const int g = R3_G, Np = N + 2 * g, N2 = N * N;
    const size_t Np2 = (size_t)Np * Np;
    const double inv_h = 1. / h;
    memset(RHS, 0, sizeof(double) * 4 * (size_t)N2);
    for (int k = 0; k < N2; k++) {
        int j = k / N, i = k % N, jp = j + g, ip = i + g;
        int kR = j * N + ((i + 1 < N) ? (i + 1) : 0);
        int kT = ((j + 1 < N) ? (j + 1) : 0) * N + i;
        ptrdiff_t b = (ptrdiff_t)jp * Np + ip;
        double F[4], G[4];
        r3_face(Q, Np2, b, 1, cx, F);
        for (int q = 0; q < 4; q++) {
            RHS[(size_t)q * N2 + k] += -F[q] * inv_h;
            RHS[(size_t)q * N2 + kR] += F[q] * inv_h;
        }
        r3_face(Q, Np2, b, Np, cy, G);
        for (int q = 0; q < 4; q++) {
            RHS[(size_t)q * N2 + k] += -G[q] * inv_h;
            RHS[(size_t)q * N2 + kT] += G[q] * inv_h;
        }
        double W[4];
        r3_w(Q[b], Q[Np2 + b], Q[2 * Np2 + b], Q[3 * Np2 + b], W);
        lam[k] = fabs(W[1]) + fabs(W[2]) + r3_snd(W[0], W[3]);
    }
}

/* 2x2-block Zhang-Shu positivity limiter (block corners by bilinear
 * extrapolation, common theta: linear for rho, 30-step bisection for p);
 * returns the number of blocks whose mean itself needed the brutal fix
 *                                              fv_rec3_2d.cu:250-337 */
int orc_rec3_limit(double *Qp, int N)
{
    const int g = R3_G, Np = N + 2 * g, Nb = N / 2;
    const size_t Np2 = (size_t)Np * Np;
    int brutal = 0;
    for (int kb = 0; kb < Nb * Nb; kb++) {
        int jb = kb / Nb, ib = kb % Nb, i0 = 2 * ib + g, j0 = 2 * jb + g;
        double U[4][4], Ub[4] = { 0., 0., 0., 0. };
        for (int c = 0; c < 4; c++) {
            int ip = i0 + (c & 1), jp = j0 + (c >> 1);
            for (int q = 0; q < 4; q++) {
                U[c][q] = Qp[q * Np2 + (size_t)jp * Np + ip];
                Ub[q] += 0.25 * U[c][q];
            }
        }
        double pb = r3_p(Ub);
        if (Ub[0] < R3_RHOFLOOR || pb < R3_PFLOOR) {
            brutal++;
            double rb = fmax(Ub[0], 10. * R3_RHOFLOOR);
            double Efix = (10. * R3_PFLOOR) / (R3_GAM - 1.) + 0.5 * (Ub[1] * Ub[1] + Ub[2] * Ub[2]) / rb;
            Ub[0] = rb;
            Ub[3] = fmax(Ub[3], Efix);
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
                double d = Ub[0] - C[c][0];
                if (d > 0.) th = fmin(th, (Ub[0] - R3_RHOFLOOR) / d);
            }
        if (th < 1.)
            for (int c = 0; c < 4; c++)
                for (int q = 0; q < 4; q++) {
                    U[c][q] = Ub[q] + th * (U[c][q] - Ub[q]);
                    C[c][q] = Ub[q] + th * (C[c][q] - Ub[q]);
                }
        int bad = 0;
        for (int c = 0; c < 4; c++)
            if (C[c][0] < R3_RHOFLOOR || r3_p(C[c]) < R3_PFLOOR) bad = 1;
        if (bad) {
            double lo = 0., hi = 1.;
            for (int it = 0; it < 30; it++) {
                double mid = 0.5 * (lo + hi);
                int ok = 1;
                for (int c = 0; c < 4; c++) {
                    double V[4];
                    for (int q = 0; q < 4; q++) V[q] = Ub[q] + mid * (C[c][q] - Ub[q]);
                    if (V[0] < R3_RHOFLOOR || r3_p(V) < R3_PFLOOR) { ok = 0; break; }
                }
                if (ok) lo = mid; else hi = mid;
            }
            for (int c = 0; c < 4; c++)
                for (int q = 0; q < 4; q++) U[c][q] = Ub[q] + lo * (U[c][q] - Ub[q]);
        }
        if (th < 1. || bad)
            for (int c = 0; c < 4; c++) {
                int ip = i0 + (c & 1), jp = j0 + (c >> 1);
                for (int q = 0; q < 4; q++) Qp[q * Np2 + (size_t)jp * Np + ip] = U[c][q];
            }
    }
    return brutal;
}

/* Qout = ca Qa + cb (Qb + dt RHS) on the interior  fv_rec3_2d.cu:339-353 */
static void r3_rk(double *Qout, const double *Qa, const double *Qb, const double *RHS, double ca, double cb,
                  double dt, int N)
{
    const int g = R3_G, Np = N + 2 * g, N2 = N * N;
    const size_t Np2 = (size_t)Np * Np;
    for (int k = 0; k < N2; k++) {
        int j = k / N, i = k % N;
        size_t c = (size_t)(j + g) * Np + (i + g);
        for (int q = 0; q < 4; q++)
            Qout[q * Np2 + c] = ca * Qa[q * Np2 + c] + cb * (Qb[q * Np2 + c] + dt * RHS[(size_t)q * N2 + k]);
    }
}

/* isentropic vortex of the paper, and the Gresho low-Mach vortex
 *                                              fv_rec3_2d.cu:356-381 */
static void r3_pv(double x, double y, double *ro, double *uo, double *vo, double *po)
{
    const double gg = R3_GAM, eps = 5., pi = 3.14159265358979323846;
    double dx = x - 5., dy = y - 5., r2 = dx * dx + dy * dy;
    double f = eps / (2. * pi) * exp(0.5 * (1. - r2));
    double dT = -(gg - 1.) * eps * eps / (8. * gg * pi * pi) * exp(1. - r2);
    double T = 1. + dT;
    if (T < 1e-6) T = 1e-6;
    *ro = pow(T, 1. / (gg - 1.));
    *po = pow(T, gg / (gg - 1.));
    *uo = -f * dy;
    *vo = f * dx;
}
static double r3_lmv_vphi(double r) { if (r < 0.2) return 5. * r; if (r < 0.4) return 2. - 5. * r; return 0.; }
static double r3_lmv_p(double r, double p0)
{
    if (r < 0.2) return p0 + 12.5 * r * r;
    if (r < 0.4) return p0 + 4. * log(5. * r) + 4. - 20. * r + 12.5 * r * r;
    return p0 + 4. * log(2.) - 2.;
}
static void r3_lmv(double x, double y, double p0, double *ro, double *uo, double *vo, double *po)
{
    double dx = x - 0.5, dy = y - 0.5, r = sqrt(dx * dx + dy * dy);
    double vp = r3_lmv_vphi(r), ir = (r > 1e-30) ? 1. / r : 0.;
    *ro = 1.; *uo = -vp * dy * ir; *vo = vp * dx * ir; *po = r3_lmv_p(r, p0);
}

static const double r3_gx[4] = { -0.861136311594053, -0.339981043584856, 0.339981043584856, 0.861136311594053 };
static const double r3_gw[4] = { 0.347854845137454, 0.652145154862546, 0.652145154862546, 0.347854845137454 };

/* initial cell averages: 0 circular Sod (sharp, midpoint), 1 paper vortex,
 * 2 Gresho vortex (4x4 Gauss)                  fv_rec3_2d.cu:383-416 */
void orc_rec3_ic(double *Qp, int N, double h, int icase, double p0lmv)
{
    const int g = R3_G, Np = N + 2 * g, N2 = N * N;
    const size_t Np2 = (size_t)Np * Np;
    memset(Qp, 0, sizeof(double) * 4 * Np2);
    for (int k = 0; k < N2; k++) {
        int j = k / N, i = k % N;
        double xc = (i + 0.5) * h, yc = (j + 0.5) * h;
        double Q[4] = { 0., 0., 0., 0. };
        if (icase == 0) {
            double r = sqrt((xc - 0.5) * (xc - 0.5) + (yc - 0.5) * (yc - 0.5));
            double rho = (r < 0.25) ? 10.0 : 0.125, p = (r < 0.25) ? 10.0 : 0.1;
            Q[0] = rho;
            Q[3] = p / (R3_GAM - 1.);
        } else {
            for (int a = 0; a < 4; a++)
                for (int b = 0; b < 4; b++) {
                    double x = xc + 0.5 * h * r3_gx[a], y = yc + 0.5 * h * r3_gx[b], r, u, v, p;
                    if (icase == 1) r3_pv(x, y, &r, &u, &v, &p);
                    else r3_lmv(x, y, p0lmv, &r, &u, &v, &p);
                    double w = 0.25 * r3_gw[a] * r3_gw[b];
                    Q[0] += w * r; Q[1] += w * r * u; Q[2] += w * r * v;
                    Q[3] += w * (p / (R3_GAM - 1.) + 0.5 * r * (u * u + v * v));
                }
        }
        for (int q = 0; q < 4; q++) Qp[q * Np2 + (size_t)(j + g) * Np + (i + g)] = Q[q];
    }
}

/* L2 errors of rho and velocity against exact cell averages, summed in
 * cell order                                   fv_rec3_2d.cu:418-448 */
void orc_rec3_err(const double *Qp, int N, double h, int icase, double p0lmv, double out[2])
{
    const int g = R3_G, Np = N + 2 * g, N2 = N * N;
    const size_t Np2 = (size_t)Np * Np;
    double s1 = 0., s2 = 0.;
    for (int k = 0; k < N2; k++) {
        int j = k / N, i = k % N;
        double xc = (i + 0.5) * h, yc = (j + 0.5) * h, re = 0., rue = 0., rve = 0.;
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                double x = xc + 0.5 * h * r3_gx[a], y = yc + 0.5 * h * r3_gx[b], r, u, v, p;
                if (icase == 1) r3_pv(x, y, &r, &u, &v, &p);
                else r3_lmv(x, y, p0lmv, &r, &u, &v, &p);
                double w = 0.25 * r3_gw[a] * r3_gw[b];
                re += w * r; rue += w * r * u; rve += w * r * v;
            }
        size_t c = (size_t)(j + g) * Np + (i + g);
        double rho = Qp[c];
        double du = Qp[Np2 + c] / rho - rue / re, dv = Qp[2 * Np2 + c] / rho - rve / re;
        s1 += (rho - re) * (rho - re) * h * h;
        s2 += (du * du + dv * dv) * h * h;
    }
    out[0] = sqrt(s1);
    out[1] = sqrt(s2);
}

/* time loop of fv_rec3_2d.cu:551-590 on an initial state that has had its
 * limiter pass and ghost fill (as main does after ic_kernel, :542-543);
 * info: {t, steps, lam_max, last dt, brutal fixes}                          */
int orc_rec3_run(double *U, int N, double h, double cfl, int max_steps, double t_stop, double info[5])
{
    const int g = R3_G, Np = N + 2 * g;
    const size_t nP = (size_t)4 * Np * Np, n1 = (size_t)N * N;
    double *U0 = (double *)malloc(sizeof(double) * nP), *U1 = (double *)malloc(sizeof(double) * nP);
    double *L = (double *)malloc(sizeof(double) * 4 * n1), *lam = (double *)malloc(sizeof(double) * n1);
    memcpy(U1, U, sizeof(double) * nP);
    orc_rec3_rhs(U, L, lam, N, h);
    double lmax = orc_max_f64(lam, n1), t = 0., dt = 0.;
    int step = 0, status = 0, brutal = 0;
    while (step < max_steps && t < t_stop) {
        if (!(lmax > 0.)) { status = 1; break; }
        dt = cfl * h / lmax;
        if (t + dt > t_stop) dt = t_stop - t;
        if (dt < 1e-14) { status = 2; break; }
        memcpy(U0, U, sizeof(double) * nP);
        r3_rk(U1, U0, U0, L, 0., 1., dt, N);
        brutal += orc_rec3_limit(U1, N);
        orc_bc_f64(U1, N, g, 1);
        orc_rec3_rhs(U1, L, lam, N, h);
        r3_rk(U1, U0, U1, L, 0.75, 0.25, dt, N);
        brutal += orc_rec3_limit(U1, N);
        orc_bc_f64(U1, N, g, 1);
        orc_rec3_rhs(U1, L, lam, N, h);
        r3_rk(U, U0, U1, L, 1. / 3., 2. / 3., dt, N);
        brutal += orc_rec3_limit(U, N);
        orc_bc_f64(U, N, g, 1);
        orc_rec3_rhs(U, L, lam, N, h);
        lmax = orc_max_f64(lam, n1);
        t += dt;
        step++;
    }
    if (info) { info[0] = t; info[1] = step; info[2] = lmax; info[3] = dt; info[4] = brutal; }
    free(U0); free(U1); free(L); free(lam);
    return status;
}

/* single-face entry points for the unit checks */
void orc_rec3_hllc(const double L[4], const double R[4], double F[4]) { r3_hllc(L, R, F); }
void orc_rec3_scale(const double Ub[4], double U[4]) { r3_scale(Ub, U); }
