// fvb_aux.cu -- the kernels around the stage kernel: ghost-ring fill,
// initial states, layout conversion between the caller's IDX_P arrays and
// the internal pitched buffers, the max-wave-speed reduction of a fresh
// state, FP64 conserved sums, and the reference's pointwise kernels
// (rk3_sX, reduce_max) for the kernel-level contract.
#include <math.h>

#include "fvb_aux.h"
#include "fvb_physics.cuh"

namespace fvb {

// row j and column i of cell k of an n x n grid (k = j n + i): a 32-bit
// unsigned division while k fits, the 64-bit one only beyond
__device__ __forceinline__ void cell_rc(long long k, int n, int &j, int &i)
{
    if (k <= 0xffffffffll) {
        const unsigned u = (unsigned)k, jj = u / (unsigned)n;
        j = (int)jj;
        i = (int)(u - jj * (unsigned)n);
    } else {
        j = (int)(k / n);
        i = (int)(k - (long long)j * n);
    }
}

// ---------------------------------------------------------------------------
// ghost ring
// ---------------------------------------------------------------------------
__device__ __forceinline__ int src_coord(int p, int n, int g, int bc, bool &ghost)
{
    // padded coordinate p of a ghost -> padded coordinate of its source
    ghost = (p < g || p >= n + g);
    if (!ghost) return p;
    if (bc == FVB_BC_REFLECT) return p < g ? 2 * g - 1 - p : 2 * (n + g) - 1 - p;
    if (bc == FVB_BC_PERIODIC) return p < g ? p + n : p - n;
    return p < g ? g : n + g - 1;
}

// Fill every ghost cell of a padded buffer from the interior cell it mirrors
// (reflect: fv_up7_ducros_2d.cu:338-362, periodic: keep_fv_euler_2d.cu:224-243,
// transmissive: zero-gradient).  One thread per ghost cell: the ring is
// enumerated as the g bottom rows, the g top rows, then the left and right
// g-wide column bands of the interior rows.
template <class R>
__global__ void bc_fill_kernel(R *buf, BufView v, int bcx, int bcy)
{
    const int n = v.n, g = v.g, np = n + 2 * g;
    const long long band = (long long)g * np, side = (long long)g * n;
    const long long total = 2 * band + 2 * side;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total;
         k += (long long)blockDim.x * gridDim.x) {
        int jp, ip;
        if (k < band) { jp = (int)(k / np); ip = (int)(k % np); }
        else if (k < 2 * band) { long long m = k - band; jp = n + g + (int)(m / np); ip = (int)(m % np); }
        else {
            long long m = k - 2 * band;
            bool right = m >= side;
            if (right) m -= side;
            jp = g + (int)(m / g);
            ip = (right ? n + g : 0) + (int)(m % g);
        }
        bool gx, gy;
        int ir = src_coord(ip, n, g, bcx, gx), jr = src_coord(jp, n, g, bcy, gy);
        long long d = (long long)jp * v.pitch + ip + v.xoff, s = (long long)jr * v.pitch + ir + v.xoff;
        for (int q = 0; q < 4; ++q) {
            R x = buf[s + q * v.plane];
            if (q == 1 && gx && bcx == FVB_BC_REFLECT) x = -x;
            if (q == 2 && gy && bcy == FVB_BC_REFLECT) x = -x;
            buf[d + q * v.plane] = x;
        }
    }
}

template <class R>
cudaError_t bc_fill(R *buf, const BufView &v, int bcx, int bcy, cudaStream_t s)
{
    long long total = 2LL * v.g * (v.n + 2 * v.g) + 2LL * v.g * v.n;
    int blocks = (int)((total + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    bc_fill_kernel<R><<<blocks, 256, 0, s>>>(buf, v, bcx, bcy);
    return cudaGetLastError();
}
template cudaError_t bc_fill<float>(float *, const BufView &, int, int, cudaStream_t);
template cudaError_t bc_fill<double>(double *, const BufView &, int, int, cudaStream_t);

// ---------------------------------------------------------------------------
// initial states: primitives in FP64 into a (4, n, n) staging array
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// uniform in [0, 1) from the k-th draw of the stream `seed`
__device__ __forceinline__ double unit_draw(uint64_t seed, uint64_t k)
{
    return (double)(splitmix64(seed * 0x9E3779B97F4A7C15ull + k) >> 11) * 0x1.0p-53;
}

__global__ void ic_kernel(double *out, int n, double x0, double y0, double h, double gam, fvb_case c)
{
    const long long n2 = (long long)n * n;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n2;
         k += (long long)blockDim.x * gridDim.x) {
        int j, i;
        cell_rc(k, n, j, i);
        const double x = x0 + (i + 0.5) * h, y = y0 + (j + 0.5) * h;
        double r = 1, u = 0, v = 0, p = 1;
        switch (c.kind) {
        case FVB_CASE_SOD: {
            // circular Sod, tanh-smoothed over one cell (fv_up7_ducros_2d.cu:629-637)
            double rr = sqrt((x - c.param[0]) * (x - c.param[0]) + (y - c.param[1]) * (y - c.param[1]));
            double phi = 0.5 * (1. + tanh((c.param[2] - rr) / (1.0 * h)));
            r = c.param[3] + (c.param[4] - c.param[3]) * phi;
            p = c.param[5] + (c.param[6] - c.param[5]) * phi;
            break;
        }
        case FVB_CASE_VORTEX: {
            // isentropic vortex with mean flow (rt_dg_euler_2d.cu:1334-1356)
            const double beta = c.param[0], pi = 3.14159265358979323846;
            double dx = x - c.param[3], dy = y - c.param[4], r2 = dx * dx + dy * dy;
            double f = beta / (2. * pi) * exp(0.5 * (1. - r2));
            double T = 1. - (gam - 1.) * beta * beta / (8. * gam * pi * pi) * exp(1. - r2);
            if (T < 1e-6) T = 1e-6;
            r = pow(T, 1. / (gam - 1.));
            p = pow(T, gam / (gam - 1.));
            u = c.param[1] - f * dy;
            v = c.param[2] + f * dx;
            break;
        }
        case FVB_CASE_KH: {
            // double shear layer: rho_in / u_in for |y - yc| < w, seeded noise on v
            bool in = fabs(y - c.param[0]) < c.param[1];
            r = in ? c.param[2] : c.param[3];
            u = in ? c.param[4] : c.param[5];
            p = c.param[6];
            const double pi = 3.14159265358979323846;
            double noise = 2. * unit_draw(c.seed, (uint64_t)k) - 1.;
            v = 0.01 * sin(4. * pi * (x - x0) / (h * n)) + c.param[7] * noise;
            break;
        }
        case FVB_CASE_RIEMANN4: {
            // quadrant q = (x >= xm) + 2 (y >= ym) takes draws 4q..4q+3 of the
            // seed; the interfaces are tanh-smoothed over param[2] cells (0 =
            // sharp), as the reference smooths its own Sod jump, because the
            // unlimited UP7 scheme is not robust on sub-cell discontinuities
            double wx, wy;
            if (c.param[2] > 0) {
                wx = 0.5 * (1. + tanh((x - c.param[0]) / (c.param[2] * h)));
                wy = 0.5 * (1. + tanh((y - c.param[1]) / (c.param[2] * h)));
            } else {
                wx = x >= c.param[0] ? 1. : 0.;
                wy = y >= c.param[1] ? 1. : 0.;
            }
            const double wq[4] = {(1. - wx) * (1. - wy), wx * (1. - wy), (1. - wx) * wy, wx * wy};
            r = u = v = p = 0.;
            for (int q = 0; q < 4; ++q) {
                r += wq[q] * (0.1 + 1.9 * unit_draw(c.seed, 4 * q + 0));
                u += wq[q] * (-1. + 2. * unit_draw(c.seed, 4 * q + 1));
                v += wq[q] * (-1. + 2. * unit_draw(c.seed, 4 * q + 2));
                p += wq[q] * (0.1 + 1.9 * unit_draw(c.seed, 4 * q + 3));
            }
            break;
        }
        case FVB_CASE_KEEP_SOD: {
            // keep_fv circular Sod (keep_fv_euler_2d.cu:457-463)
            double rr = sqrt((x - 0.5) * (x - 0.5) + (y - 0.5) * (y - 0.5));
            double phi = 0.5 * (1. + tanh((0.25 - rr) / (1.0 * h)));
            r = 0.125 + (1.0 - 0.125) * phi;
            p = 0.1 + (1.0 - 0.1) * phi;
            break;
        }
        case FVB_CASE_LMV: {
            // stationary low-Mach vortex (keep_fv_euler_2d.cu:472-495)
            double eps = c.param[0], p0 = 1. / (gam * eps * eps) - 0.5;
            double dx = x - 0.5, dy = y - 0.5, rr = sqrt(dx * dx + dy * dy);
            double vp = (rr < 0.2) ? 5. * rr : (rr < 0.4) ? 2. - 5. * rr : 0.;
            double ir = (rr > 1e-30) ? 1. / rr : 0.;
            r = 1.;
            u = -vp * dy * ir;
            v = vp * dx * ir;
            p = (rr < 0.2) ? p0 + 12.5 * rr * rr
                : (rr < 0.4) ? p0 + 4. * log(5. * rr) + 4. - 20. * rr + 12.5 * rr * rr
                             : p0 + 4. * log(2.) - 2.;
            break;
        }
        default:
            r = c.param[0]; u = c.param[1]; v = c.param[2]; p = c.param[3];
        }
        out[k] = r;
        out[n2 + k] = u;
        out[2 * n2 + k] = v;
        out[3 * n2 + k] = p;
    }
}

// The circular Sod state of the FP32 form as shipped, evaluated in FP32 in
// the reference's expression order (fv_up7_ducros_2d.cu:618-639): FP32 h,
// cell centres, radius, tanhf blend, so the initial state has the bits the
// shipped solver starts from.  (4, n, n) floats, primitives.
__global__ void ic_sod32_kernel(float *out, int n, float x0, float y0, float h, float xc0, float yc0, float rad,
                                float r_out, float dr, float p_out, float dp)
{
    const long long n2 = (long long)n * n;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n2;
         k += (long long)blockDim.x * gridDim.x) {
        int j, i;
        cell_rc(k, n, j, i);
        const float xc = x0 + (i + 0.5f) * h, yc = y0 + (j + 0.5f) * h;
        const float r = sqrtf((xc - xc0) * (xc - xc0) + (yc - yc0) * (yc - yc0));
        const float delta = 1.0f * h;
        const float phi = 0.5f * (1.f + tanhf((rad - r) / delta));
        out[k] = r_out + dr * phi;
        out[n2 + k] = 0.f;
        out[2 * n2 + k] = 0.f;
        out[3 * n2 + k] = p_out + dp * phi;
    }
}

cudaError_t init_sod_prim32(float *out, int n, double x0, double y0, double length, const fvb_case &c,
                            cudaStream_t s)
{
    int blocks = (int)(((long long)n * n + 255) / 256);
    if (blocks > 8192) blocks = 8192;
    // h = 1.0f / N as the shipped solver forms it (scaled by the length)
    const float h = (float)length * (1.0f / (float)n);
    ic_sod32_kernel<<<blocks, 256, 0, s>>>(out, n, (float)x0, (float)y0, h, (float)c.param[0], (float)c.param[1],
                                           (float)c.param[2], (float)c.param[3], (float)(c.param[4] - c.param[3]),
                                           (float)c.param[5], (float)(c.param[6] - c.param[5]));
    return cudaGetLastError();
}

cudaError_t init_case_prim64(double *out, int n, double x0, double y0, double h, double gam,
                             const fvb_case &c, cudaStream_t s)
{
    int blocks = (int)(((long long)n * n + 255) / 256);
    if (blocks > 8192) blocks = 8192;
    ic_kernel<<<blocks, 256, 0, s>>>(out, n, x0, y0, h, gam, c);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// layout conversion
// ---------------------------------------------------------------------------
template <class T> __device__ __forceinline__ double ld64(const void *p, long long i)
{
    return (double)((const T *)p)[i];
}

__device__ __forceinline__ void prim_to_cons64(const double w[4], double c[4], double gam)
{
    c[0] = w[0];
    c[1] = w[0] * w[1];
    c[2] = w[0] * w[2];
    c[3] = w[3] / (gam - 1.) + 0.5 * w[0] * (w[1] * w[1] + w[2] * w[2]);
}
__device__ __forceinline__ void cons_to_prim64(const double c[4], double w[4], double gam)
{
    w[0] = c[0];
    w[1] = c[1] / c[0];
    w[2] = c[2] / c[0];
    w[3] = (gam - 1.) * (c[3] - 0.5 * (c[1] * c[1] + c[2] * c[2]) / c[0]);
}

// Caller array (ext: IDX_P padded or interior-only, prim or cons, f32/f64)
// -> internal buffer(s).  Internal kinds: prim in R (F64/F32 modes) or
// conserved hi/lo float pairs (F32C).  Only interior cells are converted;
// the ghosts are refilled afterwards.
__global__ void import_kernel(const void *src, ExtView e, void *dst, void *dst_lo, BufView v, int internal,
                              double gam)
{
    const int n = v.n;
    const long long n2 = (long long)n * n;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n2;
         k += (long long)blockDim.x * gridDim.x) {
        int j, i;
        cell_rc(k, n, j, i);
        long long es = e.interior ? k : (long long)(j + e.g) * e.np + (i + e.g);
        long long eplane = e.interior ? n2 : (long long)e.np * e.np;
        double x[4];
        for (int q = 0; q < 4; ++q)
            x[q] = e.dtype == FVB_F64 ? ld64<double>(src, es + q * eplane) : ld64<float>(src, es + q * eplane);
        long long d = (long long)(j + v.g) * v.pitch + (i + v.g) + v.xoff;
        if (internal == INT_CONS64) {
            double c[4];
            if (e.layout == FVB_LAYOUT_PRIM) prim_to_cons64(x, c, gam);
            else for (int q = 0; q < 4; ++q) c[q] = x[q];
            for (int q = 0; q < 4; ++q) ((double *)dst)[d + q * v.plane] = c[q];
        } else if (internal == INT_CONS_HILO) {
            double c[4];
            if (e.layout == FVB_LAYOUT_PRIM) prim_to_cons64(x, c, gam);
            else for (int q = 0; q < 4; ++q) c[q] = x[q];
            for (int q = 0; q < 4; ++q) {
                float hi = (float)c[q];
                ((float *)dst)[d + q * v.plane] = hi;
                ((float *)dst_lo)[d + q * v.plane] = (float)(c[q] - (double)hi);
            }
        } else {
            double w[4];
            if (e.layout == FVB_LAYOUT_CONS) cons_to_prim64(x, w, gam);
            else for (int q = 0; q < 4; ++q) w[q] = x[q];
            for (int q = 0; q < 4; ++q) {
                if (internal == INT_PRIM64) ((double *)dst)[d + q * v.plane] = w[q];
                else ((float *)dst)[d + q * v.plane] = (float)w[q];
            }
        }
    }
}

// internal -> caller array, interior cells (and, for a padded caller array,
// the ghost ring too: every padded cell is copied)
__global__ void export_kernel(const void *src, const void *src_lo, BufView v, int internal, void *dst, ExtView e,
                              double gam)
{
    const int n = v.n;
    const int span = e.interior ? n : n + 2 * v.g;
    const int off = e.interior ? v.g : 0;          // padded coordinate of the first exported cell
    const long long cnt = (long long)span * span;
    const long long eplane = e.interior ? (long long)n * n : (long long)e.np * e.np;
    const int eo = e.interior ? 0 : e.g - v.g;     // caller's padded offset of the same cell
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < cnt;
         k += (long long)blockDim.x * gridDim.x) {
        int jj, ii;
        cell_rc(k, span, jj, ii);
        const int jp = jj + off, ip = ii + off;
        long long s = (long long)jp * v.pitch + ip + v.xoff;
        double x[4];
        if (internal == INT_CONS_HILO || internal == INT_CONS64) {
            for (int q = 0; q < 4; ++q)
                x[q] = internal == INT_CONS64 ? ((const double *)src)[s + q * v.plane]
                                              : (double)((const float *)src)[s + q * v.plane] +
                                                    (double)((const float *)src_lo)[s + q * v.plane];
            if (e.layout == FVB_LAYOUT_PRIM) { double w[4]; cons_to_prim64(x, w, gam); for (int q = 0; q < 4; ++q) x[q] = w[q]; }
        } else {
            for (int q = 0; q < 4; ++q)
                x[q] = internal == INT_PRIM64 ? ((const double *)src)[s + q * v.plane] : (double)((const float *)src)[s + q * v.plane];
            if (e.layout == FVB_LAYOUT_CONS) { double c[4]; prim_to_cons64(x, c, gam); for (int q = 0; q < 4; ++q) x[q] = c[q]; }
        }
        long long d = e.interior ? k : (long long)(jj + eo) * e.np + (ii + eo);
        for (int q = 0; q < 4; ++q) {
            if (e.dtype == FVB_F64) ((double *)dst)[d + q * eplane] = x[q];
            else ((float *)dst)[d + q * eplane] = (float)x[q];
        }
    }
}

cudaError_t import_state(const void *src, const ExtView &e, void *dst, void *dst_lo, const BufView &v,
                         int internal, double gam, cudaStream_t s)
{
    int blocks = (int)(((long long)v.n * v.n + 255) / 256);
    if (blocks > 8192) blocks = 8192;
    import_kernel<<<blocks, 256, 0, s>>>(src, e, dst, dst_lo, v, internal, gam);
    return cudaGetLastError();
}

cudaError_t export_state(const void *src, const void *src_lo, const BufView &v, int internal, void *dst,
                         const ExtView &e, double gam, cudaStream_t s)
{
    long long span = e.interior ? v.n : v.n + 2 * v.g;
    int blocks = (int)((span * span + 255) / 256);
    if (blocks > 8192) blocks = 8192;
    export_kernel<<<blocks, 256, 0, s>>>(src, src_lo, v, internal, dst, e, gam);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// max wave speed of a state -> ctrl->lam_acc (the prologue of
// fv_up7_ducros_2d.cu:991-993), and FP64 conserved sums
// ---------------------------------------------------------------------------
__device__ __forceinline__ double block_max(double x, double *sh)
{
    for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = x;
    __syncthreads();
    double m = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, sh[w]);
    __syncthreads();
    return m;
}

__global__ void lam_kernel(const void *st, BufView v, int internal, double gam, unsigned long long *acc)
{
    __shared__ double sh[32];
    const int n = v.n;
    const long long n2 = (long long)n * n;
    double m = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n2;
         k += (long long)blockDim.x * gridDim.x) {
        int j, i;
        cell_rc(k, n, j, i);
        long long s = (long long)(j + v.g) * v.pitch + (i + v.g) + v.xoff;
        double lam;
        if (internal == INT_PRIM64) {
            const double *b = (const double *)st;
            Gas<double> gs{gam, gam - 1.0};
            lam = fabs(b[s + v.plane]) + fabs(b[s + 2 * v.plane]) + sound<double>(b[s + 3 * v.plane], b[s], gs);
        } else if (internal == INT_PRIM32) {
            const float *b = (const float *)st;
            Gas<float> gs{(float)gam, (float)gam - 1.0f};
            lam = fabsf(b[s + v.plane]) + fabsf(b[s + 2 * v.plane]) + sound<float>(b[s + 3 * v.plane], b[s], gs);
        } else {
            const float *b = (const float *)st;
            Gas<float> gs{(float)gam, (float)gam - 1.0f};
            float c[4] = {b[s], b[s + v.plane], b[s + 2 * v.plane], b[s + 3 * v.plane]}, w[4];
            c2p<float>(c, w, gs);
            lam = fabsf(w[1]) + fabsf(w[2]) + sound<float>(w[3], w[0], gs);
        }
        m = fmax(m, lam);
    }
    m = block_max(m, sh);
    if (threadIdx.x == 0) atomicMax(acc, (unsigned long long)__double_as_longlong(m));
}

cudaError_t lam_into(const void *st, const BufView &v, int internal, double gam, unsigned long long *acc,
                     cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(acc, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    int blocks = (int)(((long long)v.n * v.n + 255) / 256);
    if (blocks > 1184) blocks = 1184;
    lam_kernel<<<blocks, 256, 0, s>>>(st, v, internal, gam, acc);
    return cudaGetLastError();
}

// per-block partial sums of rho, rho u, rho v, E and a non-finite count;
// reduced on the host in block order (deterministic)
__global__ void sums_kernel(const void *st, const void *lo, BufView v, int internal, double gam, double *part)
{
    __shared__ double sh[5][32];
    const int n = v.n;
    const long long n2 = (long long)n * n;
    double acc[5] = {0, 0, 0, 0, 0};
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n2;
         k += (long long)blockDim.x * gridDim.x) {
        int j, i;
        cell_rc(k, n, j, i);
        long long s = (long long)(j + v.g) * v.pitch + (i + v.g) + v.xoff;
        double c[4];
        if (internal == INT_CONS64) {
            for (int q = 0; q < 4; ++q) c[q] = ((const double *)st)[s + q * v.plane];
        } else if (internal == INT_CONS_HILO) {
            for (int q = 0; q < 4; ++q)
                c[q] = (double)((const float *)st)[s + q * v.plane] + (double)((const float *)lo)[s + q * v.plane];
        } else {
            double w[4];
            for (int q = 0; q < 4; ++q)
                w[q] = internal == INT_PRIM64 ? ((const double *)st)[s + q * v.plane] : (double)((const float *)st)[s + q * v.plane];
            prim_to_cons64(w, c, gam);
        }
        bool fin = isfinite(c[0]) && isfinite(c[1]) && isfinite(c[2]) && isfinite(c[3]);
        if (fin) for (int q = 0; q < 4; ++q) acc[q] += c[q];
        else acc[4] += 1.0;
    }
    for (int q = 0; q < 5; ++q) {
        double x = acc[q];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) sh[q][threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double x = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += sh[threadIdx.x][w];
        part[blockIdx.x * 5 + threadIdx.x] = x;
    }
}

cudaError_t sums_partials(const void *st, const void *lo, const BufView &v, int internal, double gam, double *part,
                          int blocks, cudaStream_t s)
{
    sums_kernel<<<blocks, 256, 0, s>>>(st, lo, v, internal, gam, part);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// reference contract: pointwise SSP-RK3 stage (fv_up7_ducros_2d.cu:531-590)
// and max reduction (fv_up7_ducros_2d.cu:593-612)
// ---------------------------------------------------------------------------
template <class R>
__global__ void rk3_kernel(int stage, R *Uo, const R *U0, const R *Uk, const R *L, R dt, int n, int np, int g,
                           Gas<R> gs)
{
    const long long n2 = (long long)n * n, np2 = (long long)np * np;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n2;
         k += (long long)blockDim.x * gridDim.x) {
        int j, i;
        cell_rc(k, n, j, i);
        const long long c = (long long)(j + g) * np + (i + g);
        R w0[4], c0[4], cv[4], w[4];
        for (int q = 0; q < 4; ++q) w0[q] = U0[q * np2 + c];
        p2c<R>(w0, c0, gs);
        if (stage == 1) {
            for (int q = 0; q < 4; ++q) cv[q] = c0[q] + dt * L[q * n2 + k];
        } else {
            R wk[4], ck[4];
            for (int q = 0; q < 4; ++q) wk[q] = Uk[q * np2 + c];
            p2c<R>(wk, ck, gs);
            if (stage == 2)
                for (int q = 0; q < 4; ++q) cv[q] = FVB_LIT(R, 0.75) * c0[q] + FVB_LIT(R, 0.25) * (ck[q] + dt * L[q * n2 + k]);
            else
                for (int q = 0; q < 4; ++q)
                    cv[q] = (FVB_LIT(R, 1.) / FVB_LIT(R, 3.)) * c0[q] + (FVB_LIT(R, 2.) / FVB_LIT(R, 3.)) * (ck[q] + dt * L[q * n2 + k]);
        }
        c2p<R>(cv, w, gs);
        w[0] = floor14(w[0]);
        w[3] = floor14(w[3]);
        for (int q = 0; q < 4; ++q) Uo[q * np2 + c] = w[q];
    }
}

template <class R>
cudaError_t rk3_stage_ref(int stage, R *Uo, const R *U0, const R *Uk, const R *L, R dt, int n, int np, int g,
                          double gam, cudaStream_t s)
{
    int blocks = (int)(((long long)n * n + 255) / 256);
    if (blocks > 8192) blocks = 8192;
    Gas<R> gs{R(gam), R(gam) - R(1)};
    rk3_kernel<R><<<blocks, 256, 0, s>>>(stage, Uo, U0, Uk, L, dt, n, np, g, gs);
    return cudaGetLastError();
}
template cudaError_t rk3_stage_ref<float>(int, float *, const float *, const float *, const float *, float, int, int,
                                          int, double, cudaStream_t);
template cudaError_t rk3_stage_ref<double>(int, double *, const double *, const double *, const double *, double,
                                           int, int, int, double, cudaStream_t);

// max from 0 with fmax (NaN skipped); the result is atomically max-ed into
// *out as a non-negative bit pattern, *out cleared first by the caller
template <class R, class U>
__global__ void max_kernel(const R *x, size_t n, U *out)
{
    __shared__ double sh[32];
    double m = 0.0;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)blockDim.x * gridDim.x)
        m = fmax(m, (double)x[k]);
    m = block_max(m, sh);
    if (threadIdx.x == 0) {
        if (sizeof(R) == 8) atomicMax((unsigned long long *)out, (unsigned long long)__double_as_longlong(m));
        else atomicMax((unsigned int *)out, (unsigned int)__float_as_int((float)m));
    }
}

cudaError_t max_ref(const void *x, size_t n, void *out, int dtype, cudaStream_t s)
{
    size_t bytes = dtype == FVB_F64 ? 8 : 4;
    cudaError_t e = cudaMemsetAsync(out, 0, bytes, s);
    if (e != cudaSuccess) return e;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 1184) blocks = 1184;
    if (blocks < 1) blocks = 1;
    if (dtype == FVB_F64) max_kernel<double, unsigned long long><<<blocks, 256, 0, s>>>((const double *)x, n, (unsigned long long *)out);
    else max_kernel<float, unsigned int><<<blocks, 256, 0, s>>>((const float *)x, n, (unsigned int *)out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// step-control updates issued between steps
// ---------------------------------------------------------------------------
__global__ void ctrl_set_kernel(Ctrl *c, double t_stop, int reset, double t0, double cfl, double h)
{
    if (reset) {
        c->t = t0;
        c->dt = 0.0;
        c->step = 0;
        c->status = 0;
        c->active = 0;
        c->clamped = 0;
        c->cfl = cfl;
        c->h = h;
    }
    c->t_stop = t_stop;
}

cudaError_t ctrl_set(Ctrl *c, double t_stop, int reset, double t0, double cfl, double h, cudaStream_t s)
{
    ctrl_set_kernel<<<1, 1, 0, s>>>(c, t_stop, reset, t0, cfl, h);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// frame fields of fv_up7's composite image, from an FP32 primitive IDX_P
// array with its ghost ring: density, 6th-order vorticity (dv/dx - du/dy,
// central differences over +-3 cells; 4th-order over +-2 with the two ghost
// layers of the KEEP and rec3 families),
// the Ducros cell sensor (max over the cell's four faces of
// dp^2 / (dp^2 + 0.1 (pa + pb)^2)), |v| and pressure.  Output: 5 planes of
// n x n floats, row-major, j = 0 at the bottom.
//                                  fv_up7_ducros_2d.cu:114-133, :511-526, :800-829
// ---------------------------------------------------------------------------
__device__ __forceinline__ float frame_ducros(float pa, float pb)
{
    const float dp = pb - pa, ps = pb + pa;
    return dp * dp / (dp * dp + 0.1f * ps * ps);
}

// One thread per cell, 32 x 8 cells a block: the x-neighbours of a warp are
// one coalesced row, the y-neighbours rows a block shares through L1.
__global__ void __launch_bounds__(256) frame_kernel(const float *Q, int n, int g, int np, float h, float *out)
{
    const long long nn = (long long)n * n;
    const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
    if (i < n && j < n) {
        const long long k = (long long)j * n + i;
        const long long pl = (long long)np * np;
        auto at = [&](int q, int jp, int ip) { return Q[q * pl + (long long)jp * np + ip]; };
        const int jp = j + g, ip = i + g;
        const float p = at(3, jp, ip);
        const float sx = fmaxf(frame_ducros(p, at(3, jp, ip + 1)), frame_ducros(at(3, jp, ip - 1), p));
        const float sy = fmaxf(frame_ducros(p, at(3, jp + 1, ip)), frame_ducros(at(3, jp - 1, ip), p));
        float w = 0.0f;
        if (g >= 3) {
            // the six taps (-1, 9, -45, 45, -9, 1)/60 accumulated one fused
            // multiply-add at a time from zero, offset -3 first: the rounding
            // of the reference's loop                fv_up7_ducros_2d.cu:812-820
            const float cf[6] = {-1.f, 9.f, -45.f, 45.f, -9.f, 1.f};
            const int off[6] = {-3, -2, -1, 1, 2, 3};
            float dvdx = 0.f, dudy = 0.f;
#pragma unroll
            for (int d = 0; d < 6; ++d) {
                dvdx = fmaf(cf[d], at(2, jp, ip + off[d]), dvdx);
                dudy = fmaf(cf[d], at(1, jp + off[d], ip), dudy);
            }
            w = (dvdx - dudy) / (60.0f * h);
        } else {
            // two ghost layers (KEEP, rec3): the 4th-order central difference
            const float dvdx = at(2, jp, ip - 2) - 8.0f * at(2, jp, ip - 1) + 8.0f * at(2, jp, ip + 1) -
                               at(2, jp, ip + 2);
            const float dudy = at(1, jp - 2, ip) - 8.0f * at(1, jp - 1, ip) + 8.0f * at(1, jp + 1, ip) -
                               at(1, jp + 2, ip);
            w = (dvdx - dudy) / (12.0f * h);
        }
        const float u = at(1, jp, ip), v = at(2, jp, ip);
        out[k] = at(0, jp, ip);
        out[nn + k] = w;
        out[2 * nn + k] = fmaxf(sx, sy);
        out[3 * nn + k] = sqrtf(fmaf(u, u, v * v));
        out[4 * nn + k] = p;
    }
}

cudaError_t frame_fields(const float *prim, int n, int g, int np, double h, float *out, cudaStream_t s)
{
    frame_kernel<<<dim3((n + 31) / 32, (n + 7) / 8), dim3(32, 8), 0, s>>>(prim, n, g, np, (float)h, out);
    return cudaGetLastError();
}

}  // namespace fvb
