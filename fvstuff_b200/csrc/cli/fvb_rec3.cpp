// fvb_rec3 -- command-line drop-in for fvStuff's fv_rec3 (fv_rec3_2d.cu main,
// :509-607) on libfvb.
//
//   fvb_rec3 [N] [pv | lmv [eps]] [--cfl C] [--t-end T]
//
// rec3 reconstruction + HLLC + 2x2-block Zhang-Shu positivity limiter,
// SSP-RK3, FP64 (the reference's -Dreal=double build), periodic, N even:
// the sharp circular Sod (default), the paper's isentropic vortex on
// [0,10]^2 (pv) or the Gresho vortex with Mach number eps (lmv, default 0.1),
// to t = 1 at CFL 0.4.  Prints what the reference prints: the step count,
// the limiter's mean-fix count, the relative mass and energy drift, and the
// L2 errors of density and velocity against the initial cell averages (the
// vortices are stationary) or, for Sod, the final minimum density and
// pressure.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fvb.h"

int main(int argc, char **argv)
{
    int N = 256, icase = 0, pos = 0;
    double eps = 0.1, cfl = 0.4, t_end = 1.0;
    for (int k = 1; k < argc; ++k) {
        const char *a = argv[k];
        if (!std::strcmp(a, "--cfl") && k + 1 < argc) cfl = std::atof(argv[++k]);
        else if (!std::strcmp(a, "--t-end") && k + 1 < argc) t_end = std::atof(argv[++k]);
        else if (pos == 0) { N = std::atoi(a); ++pos; }
        else if (pos == 1) {
            if (!std::strcmp(a, "pv")) icase = 1;
            else if (!std::strcmp(a, "lmv")) icase = 2;
            ++pos;
        } else if (pos == 2 && icase == 2) { eps = std::atof(a); ++pos; }
    }
    if (N % 2) {
        std::fprintf(stderr, "N must be even (2x2 positivity blocks)\n");
        return 1;
    }
    const double L = icase == 1 ? 10.0 : 1.0, h = L / N;
    const char *cname = icase == 0 ? "circular Sod" : icase == 1 ? "paper vortex (pv)" : "Gresho (lmv)";
    std::printf("FV rec3 (unlimited) + HLLC + 2x2-block Zhang-Shu positivity\n");
    std::printf("  N=%d  h=%.5f  L=%.1f  CFL=%.2f  case=%s", N, h, L, cfl, cname);
    if (icase == 2) std::printf("  eps=%.4f", eps);
    std::printf("  [double]\n");

    fvb_config cfg;
    fvb_config_default(&cfg, N);
    cfg.flux = FVB_FLUX_REC3;
    cfg.bc_x = cfg.bc_y = FVB_BC_PERIODIC;
    cfg.length = L;
    cfg.cfl = cfl;
    fvb_solver *s = nullptr;
    if (fvb_create(&cfg, &s)) { std::fprintf(stderr, "fvb_create: %s\n", fvb_last_error()); return 1; }
    fvb_case c;
    const int kind = icase == 0 ? FVB_CASE_REC3_SOD : icase == 1 ? FVB_CASE_PAPER_VORTEX : FVB_CASE_GRESHO;
    fvb_case_default(&c, kind, 0.0, 0.0, L);
    if (icase == 2) c.param[0] = eps;
    if (fvb_init_case(s, &c)) { std::fprintf(stderr, "init: %s\n", fvb_last_error()); return 1; }

    // the initial cell averages (the exact solution of the two stationary
    // vortices) and the conserved totals
    const size_t nn = (size_t)N * N;
    std::vector<double> U0(4 * nn), U(4 * nn);
    if (fvb_get_state(s, U0.data(), FVB_LAYOUT_CONS, FVB_F64, FVB_HOST, 1)) {
        std::fprintf(stderr, "state: %s\n", fvb_last_error());
        return 1;
    }
    fvb_stats st;
    fvb_stats_sums(s, &st);
    const double m0 = st.sums[0], e0 = st.sums[3];

    const auto t0 = std::chrono::steady_clock::now();
    const fvb_status rs = fvb_advance(s, t_end, INT64_MAX, 64);
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    fvb_stats_sums(s, &st);
    if (rs == FVB_ERR_BLOWUP)
        std::fprintf(stderr, "NaN/Inf lam_max step %lld t=%.5f\n", (long long)st.steps, st.t);
    else if (rs == FVB_ERR_DT_UNDERFLOW)
        std::fprintf(stderr, "dt underflow step %lld t=%.5f\n", (long long)st.steps, st.t);
    else if (rs) { std::fprintf(stderr, "%s\n", fvb_last_error()); return 1; }
    std::printf("  Done: %lld steps  t=%.6f  wall=%.2fs\n", (long long)st.steps, st.t, wall);
    int64_t fixes = 0;
    fvb_limiter_fixes(s, &fixes);
    std::printf("  brutal mean-fix activations: %lld\n", (long long)fixes);
    std::printf("  conservation drift: mass %.3e  energy %.3e (relative)\n", std::fabs(st.sums[0] - m0) / std::fabs(m0),
                std::fabs(st.sums[3] - e0) / std::fabs(e0));

    if (fvb_get_state(s, U.data(), FVB_LAYOUT_CONS, FVB_F64, FVB_HOST, 1)) {
        std::fprintf(stderr, "state: %s\n", fvb_last_error());
        return 1;
    }
    if (icase != 0) {
        // fv_rec3_2d.cu:419-447: sum over cells of (rho - rho_e)^2 h^2 and of
        // |v - v_e|^2 h^2, v_e from the averaged momentum and density
        double s1 = 0., s2 = 0.;
        for (size_t k = 0; k < nn; ++k) {
            const double rho = U[k], re = U0[k];
            const double du = U[nn + k] / rho - U0[nn + k] / re, dv = U[2 * nn + k] / rho - U0[2 * nn + k] / re;
            s1 += (rho - re) * (rho - re) * h * h;
            s2 += (du * du + dv * dv) * h * h;
        }
        std::printf("  L2(rho) = %.6e\n", std::sqrt(s1));
        std::printf("  L2(vel) = %.6e\n", std::sqrt(s2));
    } else {
        double rmin = 1e30, pmin = 1e30;
        for (size_t k = 0; k < nn; ++k) {
            const double r = U[k], mx = U[nn + k], my = U[2 * nn + k], E = U[3 * nn + k];
            const double p = (cfg.gamma - 1.) * (E - 0.5 * (mx * mx + my * my) / r);
            rmin = std::min(rmin, r);
            pmin = std::min(pmin, p);
        }
        std::printf("  final min rho = %.4e   min p = %.4e\n", rmin, pmin);
    }
    fvb_destroy(s);
    return 0;
}
