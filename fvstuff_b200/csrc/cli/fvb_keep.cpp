// fvb_keep -- command-line drop-in for fvStuff's keep_fv (keep_fv_euler_2d.cu
// main, :594-764) on libfvb.
//
//   fvb_keep [N] [lmv [eps]] [--cfl C] [--t-end T] [--resume FILE]
//
// Circular Sod (default) or the stationary low-Mach vortex with Mach number
// eps (default 0.1) on the periodic unit square, KEEP flux (ECKEP + JST /
// MOVERS-RH), SSP-RK3, FP64; CFL 0.2; t_end 0.25 (Sod) or one vortex period
// 2 pi 0.2 (lmv); 10 frames as figures/keep_{sod,lmv}_%04d.png (left: density
// or |v|, right: pressure, jet), L2 errors of rho and p for lmv.
#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "fvb.h"
#include "fvb_io.h"

namespace {

const double kPi = 3.14159265358979323846;

// L2 errors of rho and p against the exact stationary vortex
//                                                keep_fv_euler_2d.cu:472-536
void lmv_errors(const std::vector<double> &Q, int N, double h, double eps, double gam, double &er, double &ep)
{
    const double p0 = 1. / (gam * eps * eps) - 0.5;
    const int g = 2, Np = N + 2 * g;
    const size_t P = (size_t)Np * Np;
    double sr = 0., sp = 0.;
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
            const double x = (i + 0.5) * h - 0.5, y = (j + 0.5) * h - 0.5, r = std::sqrt(x * x + y * y);
            const double pe = r < 0.2 ? p0 + 12.5 * r * r
                                      : r < 0.4 ? p0 + 4. * std::log(5. * r) + 4. - 20. * r + 12.5 * r * r
                                                : p0 + 4. * std::log(2.) - 2.;
            const size_t c = (size_t)(j + g) * Np + (i + g);
            const double rho = std::fmax(Q[c], 1e-14), u = Q[P + c] / rho, v = Q[2 * P + c] / rho;
            const double p = (gam - 1.) * (Q[3 * P + c] - 0.5 * rho * (u * u + v * v));
            sr += (rho - 1.) * (rho - 1.) * h * h;
            sp += (p - pe) * (p - pe) * h * h;
        }
    er = std::sqrt(sr);
    ep = std::sqrt(sp);
}

}  // namespace

int main(int argc, char **argv)
{
    int N = 200;
    bool lmv = false;
    double eps = 0.1, cfl = 0.2, t_end = -1.0;
    std::string resume;
    int pos = 0;
    for (int k = 1; k < argc; ++k) {
        std::string s = argv[k];
        if (s == "--cfl" && k + 1 < argc) cfl = std::atof(argv[++k]);
        else if (s == "--t-end" && k + 1 < argc) t_end = std::atof(argv[++k]);
        else if (s == "--resume" && k + 1 < argc) resume = argv[++k];
        else if (pos == 0) { N = std::atoi(s.c_str()); ++pos; }
        else if (pos == 1) { lmv = (s == "lmv"); ++pos; }
        else if (pos == 2 && lmv) {
            char *end;
            double m = std::strtod(s.c_str(), &end);
            if (end != s.c_str() && *end == '\0' && m > 0.) eps = m;
            ++pos;
        }
    }
    if (t_end <= 0) t_end = lmv ? 2. * kPi * 0.2 : 0.25;
    const double gam = 1.4, h = 1.0 / N;
    fvb_config cfg;
    fvb_config_default(&cfg, N);
    cfg.flux = FVB_FLUX_KEEP;
    cfg.bc_x = cfg.bc_y = FVB_BC_PERIODIC;
    cfg.cfl = cfl;
    fvb_solver *s = nullptr;
    if (fvb_create(&cfg, &s)) { std::fprintf(stderr, "fvb_create: %s\n", fvb_last_error()); return 1; }
    std::printf("========================================================\n");
    const char *dev_name = fvb_device_name(cfg.device);
    std::printf("  Device : %s\n", dev_name ? dev_name : fvb_version());
    std::printf("  Collocated FV + KEEP (ECKEP+ES, eq.41)  --  %s\n", lmv ? "Low-Mach Vortex" : "Circular Sod");
    if (lmv) std::printf("  eps=%.4f  (p0=%.3f)\n", eps, 1. / (gam * eps * eps) - 0.5);
    std::printf("  N=%dx%d  Np=%d  h=%.5f  CFL=%.2f  t_end=%.4f\n", N, N, N + 4, h, cfl, t_end);
    std::printf("  DOFs: rho, rho*u, rho*v, E  (collocated P0, no enriched DOFs)\n");
    std::printf("========================================================\n");
    fvb_case c;
    fvb_case_default(&c, lmv ? FVB_CASE_LMV : FVB_CASE_KEEP_SOD, 0, 0, 1);
    if (lmv) c.param[0] = eps;
    if (fvb_init_case(s, &c)) { std::fprintf(stderr, "init: %s\n", fvb_last_error()); return 1; }
    // continue from a checkpoint (fvb_save) of a solver of this configuration
    if (!resume.empty() && fvb_load(s, resume.c_str())) {
        std::fprintf(stderr, "resume: %s\n", fvb_last_error());
        return 1;
    }

    const int Np = N + 4;
    std::vector<double> Q((size_t)4 * Np * Np);
    std::vector<unsigned char> img((size_t)3 * 2 * N * N);
    const char *prefix = lmv ? "keep_lmv" : "keep_sod";
    mkdir("figures", 0755);
    auto frame = [&](int idx) {
        fvb_get_state(s, Q.data(), FVB_LAYOUT_CONS, FVB_F64, FVB_HOST, 0);
        const size_t P = (size_t)Np * Np;
        std::vector<double> L((size_t)N * N), R((size_t)N * N);
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) {
                const size_t cc = (size_t)(j + 2) * Np + (i + 2), k = (size_t)j * N + i;
                const double rho = std::fmax(Q[cc], 1e-14), mx = Q[P + cc], my = Q[2 * P + cc];
                const double u = mx / rho, v = my / rho;
                L[k] = lmv ? std::sqrt(mx * mx + my * my) / rho : rho;
                R[k] = (gam - 1.) * (Q[3 * P + cc] - 0.5 * rho * (u * u + v * v));
            }
        const double Lhi = std::max(*std::max_element(L.begin(), L.end()), 1e-12);
        auto rm = std::minmax_element(R.begin(), R.end());
        const double Rlo = *rm.first, Rhi = *rm.second;
        for (int r = 0; r < N; ++r)
            for (int cx = 0; cx < 2 * N; ++cx) {
                const int pj = N - 1 - r, ci = cx < N ? cx : cx - N;
                const double v = (cx < N ? L : R)[(size_t)pj * N + ci];
                const double lo = cx < N ? 0. : Rlo, hi = cx < N ? Lhi : Rhi;
                double t = (v - lo) / (hi - lo + 1e-30);
                if (!(t > 0.)) t = 0.;
                if (t > 1.) t = 1.;
                fvbio::RGB px = fvbio::jet(t);
                unsigned char *o = img.data() + ((size_t)r * 2 * N + cx) * 3;
                o[0] = px.r; o[1] = px.g; o[2] = px.b;
            }
        char fn[128];
        std::snprintf(fn, sizeof fn, "figures/%s_%04d.png", prefix, idx);
        if (fvbio::write_png(fn, img.data(), 2 * N, N)) std::printf("  Saved %s\n", fn);
        if (lmv) {
            double er, ep;
            lmv_errors(Q, N, h, eps, gam, er, ep);
            std::printf("    L2_rho=%.4e  L2_p=%.4e\n", er, ep);
        }
    };
    const int NF = 10;
    int f = 1;
    fvb_stats st;
    fvb_sync(s, &st);
    // a resumed run starts at the first frame after its time
    if (st.t == 0.0) frame(0);
    else while (f <= NF && st.t >= f * t_end / NF - 1e-12) ++f;
    double t_next = f * t_end / NF;
    const auto t0 = std::chrono::steady_clock::now();
    while (st.t < t_end) {
        if (fvb_step(s, 50, std::min(t_next, t_end)) || fvb_sync(s, &st)) { std::fprintf(stderr, "%s\n", fvb_last_error()); return 1; }
        // the reference's two stops               keep_fv_euler_2d.cu:701-705
        if (st.status == FVB_ERR_BLOWUP) { std::fprintf(stderr, "NaN lam at step %lld\n", (long long)st.steps); break; }
        if (st.status) { std::fprintf(stderr, "dt underflow\n"); break; }
        if (st.t >= t_next - 1e-12 && f <= NF) {
            const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            std::printf("  frame %2d/%d  step %5lld  t=%.5f  lam=%.3e  elapsed=%.1fs\n", f, NF, (long long)st.steps, st.t,
                        st.lam_max, el);
            std::fflush(stdout);
            frame(f);
            ++f;
            t_next = f * t_end / NF;
        }
    }
    if (lmv) {
        fvb_get_state(s, Q.data(), FVB_LAYOUT_CONS, FVB_F64, FVB_HOST, 0);
        double er, ep;
        lmv_errors(Q, N, h, eps, gam, er, ep);
        // the reference's report block             keep_fv_euler_2d.cu:739-747
        std::printf("  \u2500\u2500 FINAL L2 ERRORS (Low-Mach Vortex) "
                    "\u2500\u2500\u2500\u2500\u2500\u2500\u2500\u2500\u2500\u2500\u2500\u2500\u2500\u2500\u2500\u2500\n");
        std::printf("  eps=%.4f  N=%d  h=%.5f  t=%.4f\n", eps, N, h, st.t);
        std::printf("  L2(rho) = %.6e\n  L2(p)   = %.6e\n", er, ep);
        std::printf("  ");
        for (int k = 0; k < 53; ++k) std::printf("\u2500");
        std::printf("\n");
    }
    const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("  Done: %lld steps  t=%.6f  wall=%.2fs\n", (long long)st.steps, st.t, wall);
    std::printf("  Output: figures/%s_0000.png .. figures/%s_%04d.png\n", prefix, prefix, NF);
    std::printf("  Left panel: %s   Right panel: pressure  (jet)\n", lmv ? "|velocity|" : "density");
    fvb_destroy(s);
    return 0;
}
