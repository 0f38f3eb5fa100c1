// fvb_up7 -- command-line drop-in for fvStuff's fv_up7 (fv_up7_ducros_2d.cu
// main, :886-1067) on libfvb.
//
//   fvb_up7 [N] [--cfl C] [--t-end T] [--case sod|vortex|kh|riemann4]
//           [--gamma G] [--bc reflect|periodic|transmissive] [--order 3|5|7|9]
//           [--precision f64|f32|f32c] [--frames F] [--prefix P] [--seed S]
//           [--bin] [--no-ppm] [--save FILE] [--resume FILE]
//           [--metrics FILE] (JSON lines: per frame, blow-up and the end)
//   fvb_up7 --d2av [N [C2 [Cg [sc [order]]]]] [options above]
//
// Defaults are the reference's: N = 400, CFL 0.40, t_end 1, circular Sod
// with reflecting walls on [0,1]^2, UP7 (FP64 arithmetic here), 10 frames
// written as <prefix>_%04d.ppm (2N x 2N composite: density, vorticity,
// Ducros sensor, |v|), frame 99 on blow-up.
//
// --d2av runs the scheme kept in fv_up7_ducros_2d.cu.bak instead (UP-order
// reconstruction of the conserved variables, HLLC, Ducros-gated D2
// viscosity), with that file's positional arguments (:741-745: N, C2, Cg,
// sc, order; defaults 400, 0.5, 0, 0.05, 5), its Sod (density 10 inside)
// and its composite, whose sensor panel is the velocity-divergence weight.
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

struct Args {
    int n = 400, order = 7, frames = 10, precision = FVB_PREC_F64, bc = -1, kase = FVB_CASE_SOD;
    double cfl = 0.40, t_end = 1.0, gamma = 1.4;
    long long seed = -1;
    std::string prefix = "sod", save, resume, metrics;
    bool bin = false, ppm = true;
    bool d2av = false;
    double c2 = 0.5, cg = 0.0, sc = 0.05;
};

int parse_enum(const char *v, const char *const *names, int count, const char *what)
{
    for (int k = 0; k < count; ++k)
        if (!std::strcmp(v, names[k])) return k;
    std::fprintf(stderr, "unknown %s '%s'\n", what, v);
    std::exit(2);
}

Args parse(int argc, char **argv)
{
    static const char *cases[] = {"sod", "vortex", "kh", "riemann4"};
    static const char *bcs[] = {"reflect", "periodic", "transmissive"};
    static const char *precs[] = {"f64", "f32", "f32c"};
    Args a;
    for (int k = 1; k < argc; ++k)
        if (!std::strcmp(argv[k], "--d2av")) { a.d2av = true; a.order = 5; }
    int npos = 0;
    for (int k = 1; k < argc; ++k) {
        std::string s = argv[k];
        auto val = [&]() -> const char * {
            if (k + 1 >= argc) { std::fprintf(stderr, "%s needs a value\n", s.c_str()); std::exit(2); }
            return argv[++k];
        };
        if (s == "--cfl") a.cfl = std::atof(val());
        else if (s == "--t-end") a.t_end = std::atof(val());
        else if (s == "--case") a.kase = parse_enum(val(), cases, 4, "case");
        else if (s == "--gamma") a.gamma = std::atof(val());
        else if (s == "--bc") a.bc = parse_enum(val(), bcs, 3, "boundary condition");
        else if (s == "--order") a.order = std::atoi(val());
        else if (s == "--precision") a.precision = parse_enum(val(), precs, 3, "precision");
        else if (s == "--frames") a.frames = std::atoi(val());
        else if (s == "--prefix") a.prefix = val();
        else if (s == "--seed") a.seed = std::atoll(val());
        else if (s == "--bin") a.bin = true;
        else if (s == "--no-ppm") a.ppm = false;
        else if (s == "--save") a.save = val();
        else if (s == "--resume") a.resume = val();
        else if (s == "--metrics") a.metrics = val();
        else if (s == "--d2av") continue;
        else if (s[0] != '-' && !a.d2av) a.n = std::atoi(s.c_str());
        else if (s[0] != '-') {
            // the .bak's positional arguments  fv_up7_ducros_2d.cu.bak:741-745
            switch (npos++) {
            case 0: a.n = std::atoi(s.c_str()); break;
            case 1: a.c2 = std::atof(s.c_str()); break;
            case 2: a.cg = std::atof(s.c_str()); break;
            case 3: a.sc = std::atof(s.c_str()); break;
            case 4: a.order = std::atoi(s.c_str()); break;
            default: std::fprintf(stderr, "too many arguments\n"); std::exit(2);
            }
        }
        else { std::fprintf(stderr, "unknown option %s\n", s.c_str()); std::exit(2); }
    }
    if (a.bc < 0) a.bc = (a.kase == FVB_CASE_SOD) ? FVB_BC_REFLECT : (a.kase == FVB_CASE_RIEMANN4 ? FVB_BC_TRANSMISSIVE : FVB_BC_PERIODIC);
    return a;
}

// Frame fields come from the device (fvb_frame_begin / fvb_frame_end):
// density, vorticity, Ducros cell sensor, |v|, pressure.  A frame is begun
// right after the steps that reach its time, the next steps are enqueued,
// and only then is it collected and written, so the image work on the host
// overlaps the GPU's next steps.
struct Frames {
    int N;
    float rho_lo = 0.f, rho_hi = 1.f;
    std::vector<float> buf;  // 5 x N x N
    explicit Frames(int n) : N(n), buf((size_t)5 * n * n) {}
    const float *field(int k) const { return buf.data() + (size_t)k * N * N; }
};

bool finish_frame(fvb_solver *s, Frames &F, const Args &a, int idx)
{
    if (fvb_frame_end(s, F.buf.data())) {
        std::fprintf(stderr, "frame read failed: %s\n", fvb_last_error());
        return false;
    }
    const size_t nn = (size_t)F.N * F.N;
    const float *rho = F.field(0), *vort = F.field(1), *sd = F.field(2), *vmag = F.field(3), *p = F.field(4);
    char fn[512];
    if (a.ppm) {
        float wmax = 1e-10f, vmax = 1e-10f;
        for (size_t k = 0; k < nn; ++k) {
            wmax = std::max(wmax, std::fabs(vort[k]));
            vmax = std::max(vmax, vmag[k]);
        }
        std::snprintf(fn, sizeof fn, "%s_%04d.ppm", a.prefix.c_str(), idx);
        fvbio::write_ppm_2x2(fn, {rho, F.rho_lo, F.rho_hi, fvbio::PLASMA}, {vort, -wmax, wmax, fvbio::BWR},
                             {sd, 0.f, 1.f, fvbio::HOT}, {vmag, 0.f, vmax, fvbio::VIRIDIS}, F.N);
    }
    if (a.bin) {
        std::snprintf(fn, sizeof fn, "%s_%04d.bin", a.prefix.c_str(), idx);
        fvbio::write_bin(fn, rho, p, F.N);
    }
    return true;
}

bool write_frame_now(fvb_solver *s, Frames &F, const Args &a, int idx)
{
    if (fvb_frame_begin(s)) {
        std::fprintf(stderr, "frame: %s\n", fvb_last_error());
        return false;
    }
    return finish_frame(s, F, a, idx);
}

}  // namespace

int main(int argc, char **argv)
{
    Args a = parse(argc, argv);
    fvb_config cfg;
    fvb_config_default(&cfg, a.n);
    cfg.order = a.order;
    cfg.precision = a.precision;
    if (a.d2av) cfg.flux = FVB_FLUX_UP_HLLC_D2AV;
    cfg.bc_x = cfg.bc_y = a.bc;
    cfg.cfl = a.cfl;
    cfg.gamma = a.gamma;
    if (a.kase == FVB_CASE_VORTEX) { cfg.x0 = cfg.y0 = -5.0; cfg.length = 10.0; }
    fvb_solver *s = nullptr;
    if (fvb_create(&cfg, &s)) { std::fprintf(stderr, "fvb_create: %s\n", fvb_last_error()); return 1; }
    if (a.d2av && fvb_set_d2av(s, a.c2, a.cg, a.sc)) {
        std::fprintf(stderr, "fvb_set_d2av: %s\n", fvb_last_error());
        return 1;
    }
    const int g = fvb_ghost_width(s);
    const double h = cfg.length / a.n;
    static const char *names[] = {"Circular Sod", "Isentropic vortex", "Kelvin-Helmholtz", "Four-quadrant Riemann"};
    std::printf("========================================================\n");
    const char *dev_name = fvb_device_name(cfg.device);
    std::printf("  Device  : %s\n", dev_name ? dev_name : fvb_version());
    std::printf("  UP%d+HLLC+Ducros FV 2D  --  %s\n", a.order, names[a.kase]);
    if (a.d2av)
        std::printf("  n=%dx%d  h=%.5f  C2=%.3f  Cg=%.4f  sc=%.4f  CFL=%.2f  order=%d\n", a.n, a.n, h, a.c2, a.cg, a.sc,
                    a.cfl, a.order);
    else
        std::printf("  n=%dx%d  Np=%d  h=%.5f  CFL=%.2f  order=%d\n", a.n, a.n, a.n + 2 * g, h, a.cfl, a.order);
    std::printf("========================================================\n");

    fvb_case c;
    fvb_case_default(&c, a.kase, cfg.x0, cfg.y0, cfg.length);
    if (a.seed >= 0) c.seed = (uint64_t)a.seed;
    if (a.d2av && a.kase == FVB_CASE_SOD) c.param[4] = 10.0;  // fv_up7_ducros_2d.cu.bak:484
    if (fvb_init_case(s, &c)) { std::fprintf(stderr, "init: %s\n", fvb_last_error()); return 1; }
    Frames F(a.n);
    // density colour scale fixed to the initial extremes for the whole run
    // (the reference fixes 0.125 .. 10.1 for its Sod case, :932)
    if (a.kase == FVB_CASE_SOD) { F.rho_lo = 0.125f; F.rho_hi = 10.1f; }
    else {
        if (fvb_frame_begin(s) || fvb_frame_end(s, F.buf.data())) {
            std::fprintf(stderr, "frame: %s\n", fvb_last_error());
            return 1;
        }
        auto mm = std::minmax_element(F.field(0), F.field(0) + (size_t)a.n * a.n);
        F.rho_lo = *mm.first; F.rho_hi = *mm.second;
    }
    if (!a.resume.empty()) {
        if (fvb_load(s, a.resume.c_str())) { std::fprintf(stderr, "resume: %s\n", fvb_last_error()); return 1; }
    }
    fvb_stats st;
    fvb_sync(s, &st);
    // frame times; the FP32 form keeps float time as the shipped solver does
    // (float t_next = frame * t_end / N_FRAMES, fv_up7_ducros_2d.cu:983, :1050)
    auto frame_time = [&](int f) {
        return a.precision == FVB_PREC_F32 ? (double)((float)f * (float)a.t_end / (float)a.frames)
                                           : f * a.t_end / a.frames;
    };
    const double t_end = a.precision == FVB_PREC_F32 ? (double)(float)a.t_end : a.t_end;
    int frame = 1;
    if (a.resume.empty() || st.t == 0.0) write_frame_now(s, F, a, 0);
    else while (frame <= a.frames && st.t >= frame_time(frame) - 1e-12) ++frame;
    double t_next = frame_time(frame);
    const auto t0 = std::chrono::steady_clock::now();
    auto elapsed = [&] { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    long long last_print = st.steps;
    // JSON-lines metrics: one line per frame, blow-up and the end, with the
    // throughput since the start of the loop and the HBM traffic it implies
    // (85.33 B per cell-stage with 8-byte or hi/lo words, 42.67 B in FP32)
    std::FILE *mf = a.metrics.empty() ? nullptr : std::fopen(a.metrics.c_str(), "w");
    if (!a.metrics.empty() && !mf) { std::fprintf(stderr, "cannot write %s\n", a.metrics.c_str()); return 1; }
    const long long steps0 = st.steps;
    const double bytes_cs = a.precision == FVB_PREC_F32 ? 128.0 / 3.0 : 256.0 / 3.0;
    auto metric = [&](const char *event, const fvb_stats &cur) {
        if (!mf) return;
        const double wall = elapsed(), cs = 3.0 * a.n * (double)a.n * (double)(cur.steps - steps0);
        const double rate = wall > 0 ? cs / wall : 0.0;
        std::fprintf(mf,
                     "{\"event\": \"%s\", \"n\": %d, \"order\": %d, \"precision\": \"%s\", \"step\": %lld, "
                     "\"t\": %.17g, \"dt\": %.17g, \"lam_max\": %.17g, \"wall_s\": %.6f, "
                     "\"cell_stage_per_s\": %.6g, \"hbm_gbs\": %.6g}\n",
                     event, a.n, a.order, a.precision == FVB_PREC_F64 ? "f64" : a.precision == FVB_PREC_F32 ? "f32" : "f32c",
                     (long long)cur.steps, cur.t, cur.dt, cur.lam_max, wall, rate, rate * bytes_cs / 1e9);
        std::fflush(mf);
    };
    bool enqueued = false;  // steps already on the stream (issued behind a frame)
    // at most 50 steps per call so progress prints like the reference's
    auto issue = [&](const fvb_stats &cur) {
        const int chunk = (int)(50 - (cur.steps % 50));
        return fvb_step(s, chunk, std::min(t_next, t_end)) == FVB_OK;
    };
    while (st.t < t_end) {
        if (!enqueued && !issue(st)) { std::fprintf(stderr, "%s\n", fvb_last_error()); return 1; }
        enqueued = false;
        if (fvb_sync(s, &st)) { std::fprintf(stderr, "%s\n", fvb_last_error()); return 1; }
        if (st.status) {
            // the reference's two stops: a non-positive or NaN wave-speed
            // maximum after a step (no frame), and a dt below 1e-14 (frame 99)
            //                                   fv_up7_ducros_2d.cu:1002-1007, :1030
            if (st.status == FVB_ERR_BLOWUP) {
                std::fprintf(stderr, "blow-up after step %lld t=%.5f\n", (long long)st.steps, st.t);
            } else {
                std::fprintf(stderr, "  dt underflow at step %lld t=%.6f lam_max=%.3e \u2014 writing blow-up frame\n",
                             (long long)st.steps, st.t, st.lam_max);
                write_frame_now(s, F, a, 99);
            }
            metric(st.status == FVB_ERR_BLOWUP ? "blowup" : "dt_underflow", st);
            break;
        }
        if (st.t >= t_next - 1e-12 && frame <= a.frames) {
            std::printf("  frame %2d/%d  step %5lld  t=%.5f  elapsed=%.1fs\n", frame, a.frames, (long long)st.steps,
                        st.t, elapsed());
            std::fflush(stdout);
            metric("frame", st);
            if (fvb_frame_begin(s)) { std::fprintf(stderr, "frame: %s\n", fvb_last_error()); return 1; }
            ++frame;
            t_next = frame_time(frame);
            // the next steps run on the GPU while this frame is written
            if (st.t < t_end) {
                if (!issue(st)) { std::fprintf(stderr, "%s\n", fvb_last_error()); return 1; }
                enqueued = true;
            }
            finish_frame(s, F, a, frame - 1);
        } else if (st.steps / 50 != last_print / 50) {
            const double el = elapsed();
            std::printf("  step %5lld  t=%.5f  dt=%.3e  elapsed=%.1fs  ETA=%.0fs\n", (long long)st.steps, st.t, st.dt,
                        el, st.t > 0 ? (t_end - st.t) / st.t * el : 0.0);
            std::fflush(stdout);
        }
        last_print = st.steps;
    }
    std::printf("  Done: %lld steps,  t=%.6f,  wall=%.2fs\n", (long long)st.steps, st.t, elapsed());
    metric("done", st);
    if (mf) std::fclose(mf);
    if (a.ppm) std::printf("  Frames written: %s_0000.ppm .. %s_%04d.ppm  (2x2 composite)\n", a.prefix.c_str(), a.prefix.c_str(), a.frames);
    if (!a.save.empty() && fvb_save(s, a.save.c_str())) std::fprintf(stderr, "save: %s\n", fvb_last_error());
    fvb_destroy(s);
    return 0;
}
