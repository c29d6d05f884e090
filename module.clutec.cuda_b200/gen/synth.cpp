// synth.cpp — seeded synthetic rectified stereo pairs with ground truth.
//
// Every random quantity is a pure function of (seed, stream, coordinates)
// through a SplitMix64-style hash, so a pair is identical whatever the thread
// count. Left image: 4-octave fractal value noise. Right image: forward warp of
// the left image by the left-view integer disparity field, nearer surfaces
// (larger d) win collisions, right pixels that no left pixel reaches are
// filled with fresh noise, then Gaussian noise is added and the result is
// rounded and clamped to uint8.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <omp.h>

#include "../../include/ctstereo.h"  // status codes
#include "../../include/ctsynth.h"

namespace {

inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline uint64_t hash4(uint64_t seed, uint64_t a, uint64_t b, uint64_t c) {
    return mix64(mix64(mix64(seed ^ (a * 0xD6E8FEB86659FD93ull)) ^ (b * 0xA0761D6478BD642Full)) ^
                 (c * 0xE7037ED1A0B428DBull));
}
inline double u01(uint64_t h) { return double(h >> 11) * (1.0 / 9007199254740992.0); }

// Sequential generator for scene parameters.
struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(mix64(seed ^ 0x5EED5EED5EEDull)) {}
    uint64_t next() { s = mix64(s); return s; }
    double uni(double a, double b) { return a + (b - a) * u01(next()); }
    int inti(int a, int b) { return a + int(u01(next()) * double(b - a + 1)) % (b - a + 1); }  // [a, b]
};

double value_noise(uint64_t seed, int octave, double x, double y, double cell) {
    const double gx = x / cell, gy = y / cell;
    const double fx0 = std::floor(gx), fy0 = std::floor(gy);
    const int64_t ix = int64_t(fx0), iy = int64_t(fy0);
    const double fx = gx - fx0, fy = gy - fy0;
    auto v = [&](int64_t a, int64_t b) { return u01(hash4(seed, uint64_t(octave), uint64_t(a), uint64_t(b))); };
    const double sx = fx * fx * (3.0 - 2.0 * fx), sy = fy * fy * (3.0 - 2.0 * fy);
    const double a = v(ix, iy) + (v(ix + 1, iy) - v(ix, iy)) * sx;
    const double b = v(ix, iy + 1) + (v(ix + 1, iy + 1) - v(ix, iy + 1)) * sx;
    return a + (b - a) * sy;
}

// 4-octave fractal value noise in [0, 255] (cells 32, 16, 8, 4 px; amplitude
// halves per octave), contrast-stretched around mid-grey.
void fractal_image(uint64_t seed, int W, int H, std::vector<double>& out) {
    out.resize((size_t)W * H);
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            double acc = 0.0, norm = 0.0, amp = 1.0, cell = 32.0;
            for (int o = 0; o < 4; ++o) {
                acc += amp * value_noise(seed, o, x + 0.5, y + 0.5, cell);
                norm += amp;
                amp *= 0.5;
                cell *= 0.5;
            }
            const double v = 0.5 + (acc / norm - 0.5) * 2.4;
            out[(size_t)y * W + x] = std::min(255.0, std::max(0.0, v * 255.0));
        }
}

inline double gauss(uint64_t seed, int x, int y) {
    const uint64_t h1 = hash4(seed, 0x6A55, uint64_t(x), uint64_t(y));
    const uint64_t h2 = hash4(seed, 0x6A56, uint64_t(x), uint64_t(y));
    const double u1 = std::max(u01(h1), 1e-300), u2 = u01(h2);
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

struct Rect { int x0, y0, x1, y1; };

Rect random_rect(Rng& g, int W, int H, double fmin, double fmax) {
    const int w = std::max(2, int(g.uni(fmin, fmax) * W));
    const int h = std::max(2, int(g.uni(fmin, fmax) * H));
    const int x0 = g.inti(0, std::max(0, W - w));
    const int y0 = g.inti(0, std::max(0, H - h));
    return {x0, y0, std::min(W, x0 + w), std::min(H, y0 + h)};
}

}  // namespace

extern "C" int ct_synth_pair(int32_t kind, uint64_t seed, int32_t W, int32_t H, int32_t dmax, uint8_t* left,
                             uint8_t* right, int16_t* gt_out, uint8_t* occ_out) {
    if (kind < 1 || kind > 3 || W < 2 || H < 2 || dmax < 0 || dmax > 4095) return CT_EINVAL;
    Rng g(seed ^ (uint64_t(kind) << 56));
    const size_t N = (size_t)W * H;
    std::vector<int16_t> gt(N);
    double gain = 1.0, sigma = 2.0;

    if (kind == 1) {
        const int bg = std::min(4, dmax);
        std::fill(gt.begin(), gt.end(), int16_t(bg));
        for (int i = 0; i < 8; ++i) {
            const Rect r = random_rect(g, W, H, 0.10, 0.33);
            const int d = g.inti(0, dmax);
            for (int y = r.y0; y < r.y1; ++y)
                for (int x = r.x0; x < r.x1; ++x) gt[(size_t)y * W + x] = int16_t(d);
        }
    } else if (kind == 2) {
        sigma = 3.0;
        auto plane = [&](const Rect& r, double d0, double gx, double gy) {
            const double cx = 0.5 * (r.x0 + r.x1), cy = 0.5 * (r.y0 + r.y1);
            for (int y = r.y0; y < r.y1; ++y)
                for (int x = r.x0; x < r.x1; ++x) {
                    const double d = d0 + gx * (x - cx) + gy * (y - cy);
                    gt[(size_t)y * W + x] = int16_t(std::lround(std::min(double(dmax), std::max(0.0, d))));
                }
        };
        plane({0, 0, W, H}, g.uni(0.2, 0.45) * dmax, g.uni(-0.1, 0.1), g.uni(-0.1, 0.1));
        for (int i = 0; i < 24; ++i) {
            const Rect r = random_rect(g, W, H, 0.06, 0.3);
            plane(r, g.uni(0.0, double(dmax)), g.uni(-0.1, 0.1), g.uni(-0.1, 0.1));
        }
    } else {
        sigma = 2.0;
        gain = g.uni(0.9, 1.1);
        struct G { double cx, cy, s, a; } gs[6];
        const double m = std::min(W, H);
        for (auto& q : gs) q = {g.uni(0, W), g.uni(0, H), g.uni(0.08, 0.3) * m, g.uni(0.3, 1.0)};
        std::vector<double> f(N);
        double lo = 1e300, hi = -1e300;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                double v = 0.0;
                for (const auto& q : gs) {
                    const double dx = x - q.cx, dy = y - q.cy;
                    v += q.a * std::exp(-(dx * dx + dy * dy) / (2.0 * q.s * q.s));
                }
                f[(size_t)y * W + x] = v;
                lo = std::min(lo, v); hi = std::max(hi, v);
            }
        const double sc = hi > lo ? double(dmax) / (hi - lo) : 0.0;
        for (size_t i = 0; i < N; ++i) gt[i] = int16_t(std::lround((f[i] - lo) * sc));
        for (int i = 0; i < 12; ++i) {
            const Rect r = random_rect(g, W, H, 0.05, 0.2);
            const int d = g.inti(0, dmax);
            for (int y = r.y0; y < r.y1; ++y)
                for (int x = r.x0; x < r.x1; ++x) gt[(size_t)y * W + x] = int16_t(d);
        }
    }

    const uint64_t s_left = hash4(seed, uint64_t(kind), 1, 0);
    const uint64_t s_fill = hash4(seed, uint64_t(kind), 2, 0);
    const uint64_t s_noise = hash4(seed, uint64_t(kind), 3, 0);
    std::vector<double> L, F;
    fractal_image(s_left, W, H, L);
    fractal_image(s_fill, W, H, F);

    std::vector<double> Rv(F);          // holes keep the fresh noise
    std::vector<int16_t> zb(N, -1);     // winning disparity per right pixel
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const int d = gt[(size_t)y * W + x];
            const int xr = x - d;
            if (xr < 0) continue;
            // rows are independent: only this row's entries are touched
            int16_t& z = zb[(size_t)y * W + xr];
            if (d > z) { z = int16_t(d); Rv[(size_t)y * W + xr] = L[(size_t)y * W + x]; }
        }

#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const size_t o = (size_t)y * W + x;
            if (left) left[o] = uint8_t(std::lround(L[o]));
            if (right) {
                const double v = gain * Rv[o] + sigma * gauss(s_noise, x, y);
                right[o] = uint8_t(std::lround(std::min(255.0, std::max(0.0, v))));
            }
            if (gt_out) gt_out[o] = gt[o];
            if (occ_out) {
                const int d = gt[o];
                const int xr = x - d;
                occ_out[o] = uint8_t(xr < 0 || zb[(size_t)y * W + xr] != d);
            }
        }
    return CT_OK;
}
