// fvb_io.h -- image and raw-state writers of the command-line drivers.
//
//   * 2N x 2N composite PPM of density / vorticity / Ducros sensor / |v|,
//     the frame layout of fv_up7_ducros_2d.cu:837-881;
//   * 2-panel PNG (jet) of keep_fv_euler_2d.cu:561-589, with a PNG encoder
//     of its own (stored deflate blocks, CRC-32 and Adler-32);
//   * the raw .bin frame of enriched_fv_euler_2d.cu:1386-1392 read by
//     plot_rt.py: int32 N, then N*N float32 rho, then N*N float32 p.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "fvb_cmaps.h"

namespace fvbio {

struct RGB {
    unsigned char r, g, b;
};

// black -> red -> yellow -> white                  fv_up7_ducros_2d.cu:750-755
inline RGB hot(float t)
{
    if (t < 1. / 3.) return RGB{(unsigned char)(t * 3. * 255), 0, 0};
    if (t < 2. / 3.) return RGB{255, (unsigned char)((t - 1. / 3.) * 3. * 255), 0};
    return RGB{255, 255, (unsigned char)((t - 2. / 3.) * 3. * 255)};
}
// blue -> white -> red                             fv_up7_ducros_2d.cu:785-796
inline RGB bwr(float t)
{
    if (t < 0.5) return RGB{(unsigned char)(t * 2.0 * 255), (unsigned char)(t * 2.0 * 255), 255};
    return RGB{255, (unsigned char)((1.0 - t) * 2.0 * 255), (unsigned char)((1.0 - t) * 2.0 * 255)};
}
// jet                                              keep_fv_euler_2d.cu:577-579
inline RGB jet(double t)
{
    auto c = [](double v) { return std::fmax(0., std::fmin(1., v)); };
    return RGB{(unsigned char)(c(1.5 - std::fabs(4. * t - 3.)) * 255.),
               (unsigned char)(c(1.5 - std::fabs(4. * t - 2.)) * 255.),
               (unsigned char)(c(1.5 - std::fabs(4. * t - 1.)) * 255.)};
}

enum Cmap { PLASMA = 0, VIRIDIS = 1, HOT = 2, BWR = 3 };

inline float unit(float v, float lo, float hi)
{
    float t = (v - lo) / (hi - lo + 1e-30f);
    if (!(t > 0.0f)) t = 0.0f;  // NaN too
    if (t > 1.0f) t = 1.0f;
    return t;
}

// t in [0, 1] -> colour: the 256-level tables index floor(255 t), the
// analytic maps take t itself                  fv_up7_ducros_2d.cu:869-876
inline RGB color(int cmap, float t)
{
    if (cmap == PLASMA || cmap == VIRIDIS) {
        int idx = (int)(t * 255.0f);
        if (idx < 0) idx = 0;
        if (idx > 255) idx = 255;
        const unsigned char *e = cmap == PLASMA ? kPlasma[idx] : kViridis[idx];
        return RGB{e[0], e[1], e[2]};
    }
    return cmap == HOT ? hot(t) : bwr(t);
}

struct Panel {
    const float *v;
    float lo, hi;
    int cmap;
};

// 2N x 2N composite, y up: top-left, top-right / bottom-left, bottom-right
inline bool write_ppm_2x2(const std::string &fn, const Panel &tl, const Panel &tr, const Panel &bl,
                          const Panel &br, int N)
{
    FILE *f = std::fopen(fn.c_str(), "wb");
    if (!f) { std::fprintf(stderr, "Cannot open %s\n", fn.c_str()); return false; }
    std::fprintf(f, "P6\n%d %d\n255\n", 2 * N, 2 * N);
    std::vector<unsigned char> row((size_t)6 * N);
    for (int r = 0; r < 2 * N; ++r) {
        const int pj = 2 * N - 1 - r;
        for (int c = 0; c < 2 * N; ++c) {
            const Panel &P = pj >= N ? (c < N ? tl : tr) : (c < N ? bl : br);
            const int sj = pj >= N ? pj - N : pj, si = c < N ? c : c - N;
            RGB px = color(P.cmap, unit(P.v[(size_t)sj * N + si], P.lo, P.hi));
            row[3 * c] = px.r; row[3 * c + 1] = px.g; row[3 * c + 2] = px.b;
        }
        std::fwrite(row.data(), 1, row.size(), f);
    }
    std::fclose(f);
    std::printf("  Saved %s\n", fn.c_str());
    return true;
}

// ---- PNG (RGB8, stored deflate) -------------------------------------------
inline uint32_t crc32(const unsigned char *p, size_t n, uint32_t c = 0xffffffffu)
{
    static uint32_t table[256];
    static bool init = false;
    if (!init) {
        for (uint32_t k = 0; k < 256; ++k) {
            uint32_t v = k;
            for (int b = 0; b < 8; ++b) v = (v & 1) ? 0xedb88320u ^ (v >> 1) : v >> 1;
            table[k] = v;
        }
        init = true;
    }
    for (size_t i = 0; i < n; ++i) c = table[(c ^ p[i]) & 0xff] ^ (c >> 8);
    return c;
}

inline void put_be32(std::vector<unsigned char> &o, uint32_t v)
{
    o.push_back(v >> 24); o.push_back(v >> 16); o.push_back(v >> 8); o.push_back(v);
}

inline void chunk(std::vector<unsigned char> &o, const char *type, const std::vector<unsigned char> &data)
{
    put_be32(o, (uint32_t)data.size());
    size_t start = o.size();
    o.insert(o.end(), type, type + 4);
    o.insert(o.end(), data.begin(), data.end());
    put_be32(o, crc32(o.data() + start, o.size() - start) ^ 0xffffffffu);
}

inline bool write_png(const std::string &fn, const unsigned char *rgb, int W, int H)
{
    std::vector<unsigned char> raw;
    raw.reserve((size_t)H * (3 * W + 1));
    for (int r = 0; r < H; ++r) {
        raw.push_back(0);  // filter: none
        raw.insert(raw.end(), rgb + (size_t)r * 3 * W, rgb + (size_t)(r + 1) * 3 * W);
    }
    std::vector<unsigned char> z = {0x78, 0x01};
    uint32_t a = 1, b = 0;
    for (unsigned char c : raw) { a = (a + c) % 65521u; b = (b + a) % 65521u; }
    for (size_t off = 0; off < raw.size() || off == 0;) {
        size_t len = std::min<size_t>(65535, raw.size() - off);
        bool last = off + len == raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back(len & 255); z.push_back(len >> 8);
        z.push_back(~len & 255); z.push_back((~len >> 8) & 255);
        z.insert(z.end(), raw.begin() + off, raw.begin() + off + len);
        off += len;
        if (last) break;
    }
    put_be32(z, (b << 16) | a);
    std::vector<unsigned char> png = {0x89, 'P', 'N', 'G', 0x0d, 0x0a, 0x1a, 0x0a};
    std::vector<unsigned char> ihdr;
    put_be32(ihdr, W); put_be32(ihdr, H);
    ihdr.push_back(8); ihdr.push_back(2); ihdr.push_back(0); ihdr.push_back(0); ihdr.push_back(0);
    chunk(png, "IHDR", ihdr);
    chunk(png, "IDAT", z);
    chunk(png, "IEND", {});
    FILE *f = std::fopen(fn.c_str(), "wb");
    if (!f) { std::fprintf(stderr, "Cannot open %s\n", fn.c_str()); return false; }
    bool ok = std::fwrite(png.data(), 1, png.size(), f) == png.size();
    ok = std::fclose(f) == 0 && ok;
    return ok;
}

// int32 N, N*N float32 rho, N*N float32 p (row-major, j = 0 at the bottom)
inline bool write_bin(const std::string &fn, const float *rho, const float *p, int N)
{
    FILE *f = std::fopen(fn.c_str(), "wb");
    if (!f) return false;
    int32_t n = N;
    bool ok = std::fwrite(&n, 4, 1, f) == 1 && std::fwrite(rho, 4, (size_t)N * N, f) == (size_t)N * N &&
              std::fwrite(p, 4, (size_t)N * N, f) == (size_t)N * N;
    ok = std::fclose(f) == 0 && ok;
    return ok;
}

}  // namespace fvbio
