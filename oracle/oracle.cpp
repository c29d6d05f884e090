// oracle.cpp — CPU restatement of the stereo block-matching hot path.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA kernels of
// the ctstereo library: only tests/, __graft_entry__.smoke() and the
// cpu_baseline / reference legs of bench.py load it. The product never links
// or calls it, and there is no CPU fallback in the product.
//
// Parity status: the reference (CluTec.Cuda: MSVC + CUDA 8 + sm_30, and it
// depends on the CluTec.Core 2.0 headers, which are not available) cannot be
// compiled here, and it ships no tests, fixtures or golden vectors. The
// restatement below is pinned by (1) transcription of the reference kernels
// for the parts the reference defines (census bit order and strict compare,
// SAD/AD cost, NCC normalisation and its sigma < 1 rule, strict-compare WTA,
// the cross-check rule, EDisparityId codes) and (2) hand-computed
// known-answer vectors in tests/golden/. The disparity -> pixel mapping lives
// in the missing _SDisparityConfig::MapPixelPos; it is defined here as
// x_R = x_L - d (left-to-right) and x_L = x_R + d (right-to-left).
//
// All functions are extern "C", take plain host pointers, and run row bands in
// parallel with OpenMP. Every matcher evaluates each per-pixel cost once per
// (pixel, disparity) and aggregates with running box sums, so the timed CPU
// baseline is an honest scalar implementation, not a naive one.
// Disparity outputs are int16 with -1 = invalid pixel.
//
// Build: see oracle/Makefile (g++ -O3 -fopenmp -ffp-contract=off).

#include <cstdint>
#include <cstring>
#include <cmath>
#include <vector>
#include <algorithm>
#include <omp.h>

namespace {

inline int popc64(uint64_t v) { return __builtin_popcountll(v); }
constexpr int kBand = 16;  // output rows per OpenMP work item

// Exhaustive WTA over a (2r+1)^2 box-aggregated per-pixel cost.
//
// dir = 0: left-to-right; base = left, match column xm = x - (dmin + d).
// dir = 1: right-to-left; base = right, match column xm = x + (dmin + d).
// d runs over [0, D); the disparity stored is dmin + d (the reference's
// search from xDispConfig.Min(), BlockMatcherNCC.cu:789-795).
// A pixel is valid iff its window lies inside the image (r <= x < W-r and
// r <= y < H-r); disparity d is valid for it iff the matched window lies
// inside too (xm - r >= 0 and xm + r < W). WTA scans d ascending and keeps the
// first strict minimum, so ties go to the lowest d (the reference's strict
// compares: BlockMatcherSAD1.cu:176, BlockMatcherNCC.cu:300).
// cost(x, y, xm) is the per-pixel cost of base (x, y) against match (xm, y).
// curve (optional): W*H*D bytes, aggregated cost >> curve_shift saturated at
// 255, 255 for invalid d; only written for valid pixels; index d - dmin.
template <typename CostFn>
void wta_box(int W, int H, int D, int dmin, int r, int dir, CostFn cost,
             int16_t* disp, int32_t* best_cost, uint8_t* curve, int curve_shift) {
    const int s = dir == 0 ? -1 : 1;
    const int K = 2 * r + 1;
    const int nb = (H + kBand - 1) / kBand;
#pragma omp parallel
    {
        std::vector<int32_t> colsum(W), ering((size_t)K * W), best((size_t)kBand * W);
        std::vector<int16_t> bd((size_t)kBand * W);
#pragma omp for schedule(dynamic, 1)
        for (int b = 0; b < nb; ++b) {
            const int y0 = b * kBand, y1 = std::min(H, y0 + kBand);
            const int ya = std::max(y0, r), yb = std::min(y1, H - r);
            std::fill(best.begin(), best.end(), INT32_MAX);
            std::fill(bd.begin(), bd.end(), int16_t(-1));
            auto erow = [&](int yy, int d) {
                int32_t* e = &ering[(size_t)(yy % K) * W];
                for (int x = 0; x < W; ++x) {
                    const int xm = x + s * (dmin + d);
                    e[x] = (xm >= 0 && xm < W) ? cost(x, yy, xm) : 0;
                }
                return e;
            };
            if (ya < yb) {
                for (int d = 0; d < D; ++d) {
                    std::fill(colsum.begin(), colsum.end(), 0);
                    for (int yy = ya - r; yy < ya + r; ++yy) {
                        const int32_t* e = erow(yy, d);
                        for (int x = 0; x < W; ++x) colsum[x] += e[x];
                    }
                    for (int y = ya; y < yb; ++y) {
                        const int32_t* en = erow(y + r, d);
                        for (int x = 0; x < W; ++x) colsum[x] += en[x];
                        int32_t acc = 0;
                        for (int x = 0; x < 2 * r && x < W; ++x) acc += colsum[x];
                        int32_t* bst = &best[(size_t)(y - y0) * W];
                        int16_t* bdd = &bd[(size_t)(y - y0) * W];
                        for (int x = r; x < W - r; ++x) {
                            acc += colsum[x + r];
                            const int xm = x + s * (dmin + d);
                            const bool dv = (xm - r >= 0) && (xm + r < W);
                            if (dv && acc < bst[x]) { bst[x] = acc; bdd[x] = int16_t(dmin + d); }
                            if (curve)
                                curve[((size_t)y * W + x) * D + d] =
                                    dv ? uint8_t(std::min(255, acc >> curve_shift)) : uint8_t(255);
                            acc -= colsum[x - r];
                        }
                        const int32_t* eo = &ering[(size_t)((y - r) % K) * W];
                        for (int x = 0; x < W; ++x) colsum[x] -= eo[x];
                    }
                }
            }
            for (int y = y0; y < y1; ++y)
                for (int x = 0; x < W; ++x) {
                    const bool pv = (y >= r && y < H - r && x >= r && x < W - r);
                    const size_t o = (size_t)y * W + x;
                    disp[o] = pv ? bd[(size_t)(y - y0) * W + x] : int16_t(-1);
                    if (best_cost) best_cost[o] = pv ? best[(size_t)(y - y0) * W + x] : -1;
                }
        }
    }
}

}  // namespace

extern "C" {

int or_num_threads() { return omp_get_max_threads(); }
void or_set_threads(int n) { if (n > 0) omp_set_num_threads(n); }

// ---------------------------------------------------------------------------
// Census transforms
// ---------------------------------------------------------------------------

// 3x3 census with the reference semantics (CluTec.Cuda.ImgProc/
// CensusTransform.cu:60-120): bits 7..0 = neighbours (-1,-1),(0,-1),(+1,-1),
// (-1,0),(+1,0),(-1,+1),(0,+1),(+1,+1); a bit is set iff neighbour > centre
// (strict). The 1-px border is not written (the kernel returns early, :66-69).
void or_census3x3(const uint8_t* img, int W, int H, int pitch, uint8_t* out, int out_pitch) {
#pragma omp parallel for schedule(static)
    for (int y = 1; y < H - 1; ++y) {
        for (int x = 1; x < W - 1; ++x) {
            const uint8_t c = img[y * pitch + x];
            auto P = [&](int dx, int dy) { return img[(y + dy) * pitch + (x + dx)]; };
            uint8_t v = 0;
            v |= uint8_t(0x80 * (P(-1, -1) > c));
            v |= uint8_t(0x40 * (P(0, -1) > c));
            v |= uint8_t(0x20 * (P(1, -1) > c));
            v |= uint8_t(0x10 * (P(-1, 0) > c));
            v |= uint8_t(0x08 * (P(1, 0) > c));
            v |= uint8_t(0x04 * (P(-1, 1) > c));
            v |= uint8_t(0x02 * (P(0, 1) > c));
            v |= uint8_t(0x01 * (P(1, 1) > c));
            out[y * out_pitch + x] = v;
        }
    }
}

// 9x7 census: the 64-bit generalisation of CensusTransform.cu:103-119.
// Window dx in [-4,4], dy in [-3,3]: 63 positions in raster order INCLUDING
// the centre (its bit is always 0); position k (0-based) goes to bit 62-k and
// bit 63 is 0. A bit is set iff neighbour > centre (strict). Pixels closer
// than 4 columns or 3 rows to the border get descriptor 0.
void or_census9x7(const uint8_t* img, int W, int H, int pitch, uint64_t* out, int out_pitch_elems) {
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            uint64_t v = 0;
            if (x >= 4 && x < W - 4 && y >= 3 && y < H - 3) {
                const int c = img[y * pitch + x];
                int k = 0;
                for (int dy = -3; dy <= 3; ++dy)
                    for (int dx = -4; dx <= 4; ++dx, ++k)
                        if (int(img[(y + dy) * pitch + (x + dx)]) > c) v |= (uint64_t(1) << (62 - k));
            }
            out[(size_t)y * out_pitch_elems + x] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// Matchers
// ---------------------------------------------------------------------------

// Census matcher on precomputed descriptors (W*H uint64, pitch W): cost =
// popcount(cB ^ cM) (CensusDifference, BlockMatcherNCC.cu:153-158, widened to
// 64 bits), (2r+1)^2 box, WTA.
void or_match_census_desc(const uint64_t* cb, const uint64_t* cm, int W, int H, int D, int dmin, int r, int dir,
                          int16_t* disp, int32_t* best_cost, uint8_t* curve, int curve_shift) {
    wta_box(W, H, D, dmin, r, dir,
            [&](int x, int y, int xm) { return popc64(cb[(size_t)y * W + x] ^ cm[(size_t)y * W + xm]); },
            disp, best_cost, curve, curve_shift);
}

// Census matcher from images: 9x7 census of both, then or_match_census_desc.
// dir 0 uses (base, match) = (L, R); dir 1 uses (R, L).
void or_match_census(const uint8_t* L, const uint8_t* R, int W, int H, int pitch,
                     int D, int dmin, int r, int dir, int16_t* disp, int32_t* best_cost,
                     uint8_t* curve, int curve_shift) {
    std::vector<uint64_t> cl((size_t)W * H), cr((size_t)W * H);
    or_census9x7(L, W, H, pitch, cl.data(), W);
    or_census9x7(R, W, H, pitch, cr.data(), W);
    const uint64_t* cb = dir == 0 ? cl.data() : cr.data();
    const uint64_t* cm = dir == 0 ? cr.data() : cl.data();
    or_match_census_desc(cb, cm, W, H, D, dmin, r, dir, disp, best_cost, curve, curve_shift);
}

// SAD matcher: (2r+1)^2 box of |B - M| (EvalSAD, BlockMatcherSAD1.cu:151-153),
// exhaustive WTA (the reference's coarse/fine search is a separate mode).
void or_match_sad(const uint8_t* L, const uint8_t* R, int W, int H, int pitch,
                  int D, int dmin, int r, int dir, int16_t* disp, int32_t* best_cost) {
    const uint8_t* b = dir == 0 ? L : R;
    const uint8_t* m = dir == 0 ? R : L;
    wta_box(W, H, D, dmin, r, dir,
            [&](int x, int y, int xm) { return std::abs(int(b[y * pitch + x]) - int(m[y * pitch + xm])); },
            disp, best_cost, nullptr, 0);
}

// ---------------------------------------------------------------------------
// Adaptive-window matcher, "best of 5 shifted 7x7 windows":
// A(x,y,d) = min(S(x,y), S(x-3,y), S(x+3,y), S(x,y-3), S(x,y+3)), S = 7x7 box
// SAD at disparity d. (The reference AW1 scores centre + best 2 of 4
// sub-windows, Kernel.Algo.AdaptWnd_W32H16.h:240-285, and AW2 its SAD
// min-variant, Kernel.Algo.AdaptWnd3D.h:244-300; the 5-window min is this
// build's configuration.) Left-to-right, match column x - (dmin + d) for
// d in [0, D), disparity dmin + d. Pixel valid iff 6 <= x < W-6 and
// 6 <= y < H-6; d valid iff x - dmin - d - 6 >= 0.
// Sub-pixel: d* = d + (c- - c+) / (2 (c- - 2 c0 + c+)) with c-, c0, c+ the
// AW costs at d-1, d, d+1: sub32 in FP32 (float(c- - c+) / float(2 den), then
// float(dmin + d) + that), sub64 in FP64. Skipped (sub = dmin + d) when
// d = 0, d = D-1, d+1 is invalid or den <= 0. Invalid pixels: disp -1, sub -1.
// ---------------------------------------------------------------------------
// Guided variant (MatcherUseDisparity, BlockMatcherAW1.cu:996-1180): the
// winner of pixel (x, y) is taken over disparities in [lo[y W + x], hi[y W + x]]
// only (lo > hi: no disparity); the sub-pixel neighbours c-, c+ are the costs
// at the winner - 1 and + 1 whether or not they lie in the range.
void or_match_aw_guided(const uint8_t* L, const uint8_t* R, int W, int H, int pitch, int D, int dmin,
                        const int32_t* lo, const int32_t* hi, int16_t* disp, int32_t* best_cost, float* sub32,
                        double* sub64);

void or_match_aw(const uint8_t* L, const uint8_t* R, int W, int H, int pitch, int D, int dmin,
                 int16_t* disp, int32_t* best_cost, float* sub32, double* sub64) {
    or_match_aw_guided(L, R, W, H, pitch, D, dmin, nullptr, nullptr, disp, best_cost, sub32, sub64);
}

void or_match_aw_guided(const uint8_t* L, const uint8_t* R, int W, int H, int pitch, int D, int dmin,
                        const int32_t* lo, const int32_t* hi, int16_t* disp, int32_t* best_cost, float* sub32,
                        double* sub64) {
    const int r = 3, sh = 3, ext = r + sh, K = 2 * r + 1;
    const int nb = (H + kBand - 1) / kBand;
#pragma omp parallel
    {
        const int SR = kBand + 2 * sh;  // S rows per band
        std::vector<int32_t> colsum(W), ering((size_t)K * W), S((size_t)SR * W);
        std::vector<int32_t> best((size_t)kBand * W), cm1((size_t)kBand * W), cp1((size_t)kBand * W),
            prevA((size_t)kBand * W);
        std::vector<int16_t> bd((size_t)kBand * W);
        std::vector<uint8_t> need((size_t)kBand * W);
#pragma omp for schedule(dynamic, 1)
        for (int b = 0; b < nb; ++b) {
            const int y0 = b * kBand, y1 = std::min(H, y0 + kBand);
            const int ya = std::max(y0, ext), yb = std::min(y1, H - ext);
            std::fill(best.begin(), best.end(), INT32_MAX);
            std::fill(bd.begin(), bd.end(), int16_t(-1));
            std::fill(cm1.begin(), cm1.end(), -1);
            std::fill(cp1.begin(), cp1.end(), -1);
            std::fill(prevA.begin(), prevA.end(), -1);
            std::fill(need.begin(), need.end(), 0);
            if (ya < yb) {
                const int sa = ya - sh, sb = yb + sh;  // S rows [sa, sb)
                for (int d = 0; d < D; ++d) {
                    auto erow = [&](int yy) {
                        int32_t* e = &ering[(size_t)(yy % K) * W];
                        for (int x = 0; x < W; ++x) {
                            const int xm = x - dmin - d;
                            e[x] = (xm >= 0 && xm < W) ? std::abs(int(L[yy * pitch + x]) - int(R[yy * pitch + xm]))
                                                       : 0;
                        }
                        return e;
                    };
                    std::fill(colsum.begin(), colsum.end(), 0);
                    for (int yy = sa - r; yy < sa + r; ++yy) {
                        const int32_t* e = erow(yy);
                        for (int x = 0; x < W; ++x) colsum[x] += e[x];
                    }
                    for (int ys = sa; ys < sb; ++ys) {
                        const int32_t* en = erow(ys + r);
                        for (int x = 0; x < W; ++x) colsum[x] += en[x];
                        int32_t* srow = &S[(size_t)(ys - sa) * W];
                        int32_t acc = 0;
                        for (int x = 0; x < 2 * r; ++x) acc += colsum[x];
                        for (int x = r; x < W - r; ++x) {
                            acc += colsum[x + r];
                            srow[x] = acc;
                            acc -= colsum[x - r];
                        }
                        const int32_t* eo = &ering[(size_t)((ys - r) % K) * W];
                        for (int x = 0; x < W; ++x) colsum[x] -= eo[x];
                    }
                    for (int y = ya; y < yb; ++y) {
                        const int32_t* sc = &S[(size_t)(y - sa) * W];
                        const int32_t* su = &S[(size_t)(y - sh - sa) * W];
                        const int32_t* sd = &S[(size_t)(y + sh - sa) * W];
                        const size_t ro = (size_t)(y - y0) * W;
                        for (int x = ext; x < W - ext; ++x) {
                            const bool dv = (x - dmin - d - ext >= 0);
                            int32_t a = -1;
                            if (dv) {
                                a = sc[x];
                                a = std::min(a, sc[x - sh]);
                                a = std::min(a, sc[x + sh]);
                                a = std::min(a, su[x]);
                                a = std::min(a, sd[x]);
                            }
                            const size_t o = ro + x;
                            if (need[o]) { cp1[o] = a; need[o] = 0; }
                            const bool in_range = !lo || (dmin + d >= lo[(size_t)y * W + x] &&
                                                          dmin + d <= hi[(size_t)y * W + x]);
                            if (dv && in_range && a < best[o]) {
                                best[o] = a; bd[o] = int16_t(d);
                                cm1[o] = prevA[o];
                                need[o] = 1; cp1[o] = -1;
                            }
                            prevA[o] = a;
                        }
                    }
                }
            }
            for (int y = y0; y < y1; ++y)
                for (int x = 0; x < W; ++x) {
                    const size_t o = (size_t)y * W + x, q = (size_t)(y - y0) * W + x;
                    const bool pv = (y >= ext && y < H - ext && x >= ext && x < W - ext);
                    if (!pv) {
                        disp[o] = -1;
                        if (best_cost) best_cost[o] = -1;
                        sub32[o] = -1.0f; sub64[o] = -1.0;
                        continue;
                    }
                    const int d = bd[q];  // relative; -1 if none
                    disp[o] = int16_t(d < 0 ? -1 : dmin + d);
                    if (best_cost) best_cost[o] = best[q];
                    float s32 = d < 0 ? -1.0f : float(dmin + d);
                    double s64 = d < 0 ? -1.0 : double(dmin + d);
                    if (d > 0 && d < D - 1 && cp1[q] >= 0 && cm1[q] >= 0) {
                        const int32_t cm = cm1[q], c0 = best[q], cp = cp1[q];
                        const int32_t den = cm - 2 * c0 + cp;
                        if (den > 0) {
                            const float off = float(cm - cp) / float(2 * den);
                            s32 = float(dmin + d) + off;
                            s64 = double(dmin + d) + double(cm - cp) / (2.0 * double(den));
                        }
                    }
                    sub32[o] = s32; sub64[o] = s64;
                }
        }
    }
}

// ---------------------------------------------------------------------------
// NCC matcher (BlockMatcherNCC.cu:182-336, without the uint8 quantisation of
// the score, :268-271). Window (2r+1)^2, n = (2r+1)^2, exact integer sums
// Sx, Sxx (left), Sy, Syy (right at x - d), Sxy. num = n Sxy - Sx Sy,
// vx = n Sxx - Sx^2, vy = n Syy - Sy^2 (int64). The reference sets NCC = 0
// when sigma_x sigma_y < 1 (:255-262), i.e. when vx vy < n^4. Otherwise
// score32 = float(num) / sqrtf(float(vx) * float(vy)) with IEEE-rounded ops,
// score64 = num / sqrt(vx vy) in double. Argmax over valid d with a strict
// '>' scanning d ascending (lowest d on ties). Left-to-right, right column
// x - (dmin + d), disparity dmin + d; pixel valid iff its window is inside;
// d valid iff x - dmin - d - r >= 0.
// Outputs: disp (int16, -1 invalid), best32 (FP32 score at the argmax),
// best64 (FP64 score at that same d).
// ---------------------------------------------------------------------------
// Guided variant (MatcherUseDisparity, BlockMatcherNCC.cu:980-1168): pixel
// (x, y) searches only disparities in [lo[y W + x], hi[y W + x]]; lo > hi
// means no search (the pixel gets no disparity). or_match_ncc is the
// unguided case.
void or_match_ncc_guided(const uint8_t* L, const uint8_t* R, int W, int H, int pitch, int D, int dmin, int r,
                         const int32_t* lo, const int32_t* hi, int16_t* disp, float* best32, double* best64);

void or_match_ncc(const uint8_t* L, const uint8_t* R, int W, int H, int pitch, int D, int dmin, int r,
                  int16_t* disp, float* best32, double* best64) {
    or_match_ncc_guided(L, R, W, H, pitch, D, dmin, r, nullptr, nullptr, disp, best32, best64);
}

void or_match_ncc_guided(const uint8_t* L, const uint8_t* R, int W, int H, int pitch, int D, int dmin, int r,
                         const int32_t* lo, const int32_t* hi, int16_t* disp, float* best32, double* best64) {
    const int n = (2 * r + 1) * (2 * r + 1), K = 2 * r + 1;
    const int64_t n4 = (int64_t)n * n * n * n;
    // per-pixel box sums of L, L^2, R, R^2 (independent of d)
    std::vector<int32_t> bl((size_t)W * H, 0), bll((size_t)W * H, 0), br((size_t)W * H, 0), brr((size_t)W * H, 0);
#pragma omp parallel for schedule(static)
    for (int y = r; y < H - r; ++y)
        for (int x = r; x < W - r; ++x) {
            int32_t a = 0, aa = 0, b = 0, bb = 0;
            for (int dy = -r; dy <= r; ++dy)
                for (int dx = -r; dx <= r; ++dx) {
                    const int u = L[(y + dy) * pitch + x + dx], v = R[(y + dy) * pitch + x + dx];
                    a += u; aa += u * u; b += v; bb += v * v;
                }
            const size_t o = (size_t)y * W + x;
            bl[o] = a; bll[o] = aa; br[o] = b; brr[o] = bb;
        }
    const int nb = (H + kBand - 1) / kBand;
#pragma omp parallel
    {
        std::vector<int32_t> colsum(W), ering((size_t)K * W);
        std::vector<float> b32((size_t)kBand * W);
        std::vector<double> b64((size_t)kBand * W);
        std::vector<int16_t> bd((size_t)kBand * W);
#pragma omp for schedule(dynamic, 1)
        for (int b = 0; b < nb; ++b) {
            const int y0 = b * kBand, y1 = std::min(H, y0 + kBand);
            const int ya = std::max(y0, r), yb = std::min(y1, H - r);
            std::fill(b32.begin(), b32.end(), -2.0f);
            std::fill(b64.begin(), b64.end(), 0.0);
            std::fill(bd.begin(), bd.end(), int16_t(-1));
            if (ya < yb) {
                for (int d = 0; d < D; ++d) {
                    auto erow = [&](int yy) {
                        int32_t* e = &ering[(size_t)(yy % K) * W];
                        for (int x = 0; x < W; ++x) {
                            const int xm = x - dmin - d;
                            e[x] = (xm >= 0 && xm < W) ? int(L[yy * pitch + x]) * int(R[yy * pitch + xm]) : 0;
                        }
                        return e;
                    };
                    std::fill(colsum.begin(), colsum.end(), 0);
                    for (int yy = ya - r; yy < ya + r; ++yy) {
                        const int32_t* e = erow(yy);
                        for (int x = 0; x < W; ++x) colsum[x] += e[x];
                    }
                    for (int y = ya; y < yb; ++y) {
                        const int32_t* en = erow(y + r);
                        for (int x = 0; x < W; ++x) colsum[x] += en[x];
                        int32_t acc = 0;
                        for (int x = 0; x < 2 * r; ++x) acc += colsum[x];
                        const size_t ro = (size_t)(y - y0) * W;
                        for (int x = r; x < W - r; ++x) {
                            acc += colsum[x + r];
                            if (x - dmin - d - r >= 0 &&
                                (!lo || (dmin + d >= lo[(size_t)y * W + x] && dmin + d <= hi[(size_t)y * W + x]))) {
                                const size_t o = (size_t)y * W + x, om = o - dmin - d;
                                const int64_t sx = bl[o], sxx = bll[o], sy = br[om], syy = brr[om];
                                const int64_t vx = n * sxx - sx * sx, vy = n * syy - sy * sy;
                                const int64_t num = (int64_t)n * acc - sx * sy;
                                float s32;
                                if (vx * vy < n4) s32 = 0.f;
                                else s32 = float(num) / sqrtf(float(vx) * float(vy));
                                if (s32 > b32[ro + x]) {
                                    b32[ro + x] = s32; bd[ro + x] = int16_t(dmin + d);
                                    b64[ro + x] = (vx * vy < n4) ? 0.0
                                                  : double(num) / std::sqrt(double(vx) * double(vy));
                                }
                            }
                            acc -= colsum[x - r];
                        }
                        const int32_t* eo = &ering[(size_t)((y - r) % K) * W];
                        for (int x = 0; x < W; ++x) colsum[x] -= eo[x];
                    }
                }
            }
            for (int y = y0; y < y1; ++y)
                for (int x = 0; x < W; ++x) {
                    const size_t o = (size_t)y * W + x, q = (size_t)(y - y0) * W + x;
                    const bool pv = (y >= r && y < H - r && x >= r && x < W - r);
                    disp[o] = pv ? bd[q] : int16_t(-1);
                    best32[o] = pv ? b32[q] : 0.f;
                    best64[o] = pv ? b64[q] : 0.0;
                }
        }
    }
}

// ---------------------------------------------------------------------------
// Cross-check (CrossCheckDisparityMaps.cu:63-110). Maps are int16
// disparities with -1 = invalid. For each base pixel with a valid d:
// x' = x - d (lr = 1) or x + d (lr = 0); x' outside the image ->
// inconsistent; the other map at x' must hold a valid disparity within tol of
// d, else inconsistent. Invalid base pixels are copied through.
// out: d, -1 (copied invalid) or -2 (inconsistent). range[0..1] = min / max of
// the kept disparities (INT16_MAX / -1 if none).
// ---------------------------------------------------------------------------
void or_crosscheck(const int16_t* base, const int16_t* other, int W, int H, int tol, int lr,
                   int16_t* out, int32_t* range) {
    int32_t mn = INT16_MAX, mx = -1;
#pragma omp parallel for schedule(static) reduction(min : mn) reduction(max : mx)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const size_t o = (size_t)y * W + x;
            const int d = base[o];
            if (d < 0) { out[o] = base[o]; continue; }
            const int xo = lr ? x - d : x + d;
            if (xo < 0 || xo >= W) { out[o] = -2; continue; }
            const int dr = other[(size_t)y * W + xo];
            if (dr >= 0 && std::abs(dr - d) <= tol) {
                out[o] = int16_t(d);
                mn = std::min(mn, d); mx = std::max(mx, d);
            } else {
                out[o] = -2;
            }
        }
    }
    range[0] = mn; range[1] = mx;
}

// ---------------------------------------------------------------------------
// Exhaustive check of the constant-divisor quotient the reference-compat
// kernel uses instead of an IEEE division (Markstein's remainder correction:
// q = RN(x z), r = RN(x - q d) by a fused multiply-add, q' = RN(q + r z),
// z = RN(1 / d)): counts the integers x with |x| <= nmax where q' differs
// from the IEEE quotient x / d in binary32.
// ---------------------------------------------------------------------------
long or_div_int_mismatches(int d, int nmax) {
    const float df = float(d);
    volatile float one = 1.0f;  // keeps the reciprocal a run-time IEEE division
    const float z = one / df;
    long bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
    for (long n = -long(nmax); n <= long(nmax); ++n) {
        const float x = float(n);
        const float want = x / df;
        const float q = x * z;
        const float r = std::fma(-q, df, x);
        const float q1 = std::fma(r, z, q);
        bad += (q1 != want);
    }
    return bad;
}

// ---------------------------------------------------------------------------
// Box sums of a KX x KY window anchored at its top-left pixel (x, y), for
// x <= W - KX and y <= H - KY (out is (H - KY + 1) x (W - KX + 1)), by the
// aggregation scheme of wta_box: running column sums over KY rows, then a
// running horizontal sum over KX columns (wta_box centres the window: its sum
// for centre (x, y) is this one at (x - r, y - r), KX = KY = 2r + 1). The
// reference's AlgoArraySum_W32H16 (Kernel.Algo.ArraySum_W32H16.h:94-272)
// computes the same sums per block tile in two passes of the same kind.
// ---------------------------------------------------------------------------
void or_box_sums(const int32_t* data, int W, int H, int KX, int KY, int32_t* out) {
    const int OW = W - KX + 1, OH = H - KY + 1;
    if (OW <= 0 || OH <= 0) return;
    std::vector<int32_t> colsum(W, 0);
    for (int yy = 0; yy < KY - 1; ++yy)
        for (int x = 0; x < W; ++x) colsum[x] += data[(size_t)yy * W + x];
    for (int y = 0; y < OH; ++y) {
        for (int x = 0; x < W; ++x) colsum[x] += data[(size_t)(y + KY - 1) * W + x];
        int32_t acc = 0;
        for (int x = 0; x < KX - 1; ++x) acc += colsum[x];
        for (int x = 0; x < OW; ++x) {
            acc += colsum[x + KX - 1];
            out[(size_t)y * OW + x] = acc;
            acc -= colsum[x];
        }
        for (int x = 0; x < W; ++x) colsum[x] -= data[(size_t)y * W + x];
    }
}

// ---------------------------------------------------------------------------
// Cross-check on EDisparityId codes, the reference rule exactly
// (CrossCheckDisparityMaps.cu:63-110): for a base code v in [First, Last]
// (disparity d = v - First) at an interior pixel, x' = x - d (lr = 1) or
// x + d; x' outside the image -> Inconsistent; else kept iff
// |other(x', y) - v| <= tol with other's code compared raw (an ID or Unknown
// too), otherwise Inconsistent. Other base codes are copied through.
// frame = 1: the 1-pixel image frame is not written (out keeps its values)
// and not counted (the kernel's IsInside(x, y, 1, 1) early return, :71);
// frame = 0: frame pixels are processed like the rest. range[0..1] = min /
// max of the kept codes, (Last, First) when none is kept (ResetRange and the
// host reduction, .cu:155-186).
// ---------------------------------------------------------------------------
void or_crosscheck_codes(const uint16_t* base, const uint16_t* other, int W, int H, int tol, int lr, int frame,
                         uint16_t* out, int32_t* range) {
    constexpr int kFirst = 1, kLast = 0xFFEF, kInconsistent = 0xFFFA;
    int32_t mn = kLast, mx = kFirst;
    const int f = frame ? 1 : 0;
#pragma omp parallel for schedule(static) reduction(min : mn) reduction(max : mx)
    for (int y = f; y < H - f; ++y) {
        for (int x = f; x < W - f; ++x) {
            const size_t o = (size_t)y * W + x;
            const int v = base[o];
            if (v < kFirst || v > kLast) { out[o] = uint16_t(v); continue; }
            const int xo = lr ? x - (v - kFirst) : x + (v - kFirst);
            if (xo < 0 || xo >= W) { out[o] = kInconsistent; continue; }
            if (std::abs(int(other[(size_t)y * W + xo]) - v) <= tol) {
                out[o] = uint16_t(v);
                mn = std::min(mn, v); mx = std::max(mx, v);
            } else {
                out[o] = kInconsistent;
            }
        }
    }
    range[0] = mn; range[1] = mx;
}

}  // extern "C"
