// compat.cpp — CPU restatement of the reference matchers' own output: the
// 4 x uint16 TPixelEx pixel (x = disparity + First or an EDisparityId, y =
// the score, z / w = the specificity channels) that BlockMatcherSAD1, NCC,
// AW1, AW2 and BlockMatcher1 write, with their gradient gates, score
// thresholds, saturation rules and the sequential scan bookkeeping that
// records the score next to the winner.
//
// TEST INFRASTRUCTURE ONLY (see oracle.cpp): the checker of the library's
// reference-compat kernels (csrc/compat.cu). Each step cites the reference
// lines it follows. Where the reference's behaviour depends on its thread
// block tiling (which disparities a block evaluates near the image border,
// SAD1's block-wide fine-search vote) it is restated per pixel:
//   * pixel (x, y) is evaluated iff its whole patch lies inside the image
//     (else it gets (CannotEvaluate, 0, 0, 0); the reference leaves it unwritten);
//   * disparity d is searched iff the matched patch lies inside too;
//   * SAD1's fine pass evaluates d for a pixel iff d is within 4 of that
//     pixel's current winner (the reference asks whether any pixel of its
//     block needs d).
// Float arithmetic follows the reference's operation order with IEEE
// rounding and no contraction (the Makefile passes -ffp-contract=off).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <vector>
#include <omp.h>

namespace {

constexpr uint16_t kFirst = 0x0001, kLast = 0xFFEF, kUnknown = 0x0000, kCannot = 0xFFFF, kSaturated = 0xFFFE,
                   kNotFound = 0xFFFD, kNotSpecific = 0xFFFC;

enum Method { kSad1 = 0, kNcc = 1, kAw1 = 2, kAw2 = 3, kBm1 = 4 };

// Box sums over [x - a, x + b] x [y - a, y + b] of a W x H plane (0 where the
// box leaves the plane; callers only read boxes inside).
struct Box {
    int W, H;
    std::vector<int64_t> I;  // (W + 1) x (H + 1) integral image
    Box(const int32_t* v, int W_, int H_) : W(W_), H(H_), I((size_t)(W_ + 1) * (H_ + 1), 0) {
        for (int y = 0; y < H; ++y) {
            int64_t row = 0;
            for (int x = 0; x < W; ++x) {
                row += v[(size_t)y * W + x];
                I[(size_t)(y + 1) * (W + 1) + x + 1] = I[(size_t)y * (W + 1) + x + 1] + row;
            }
        }
    }
    int64_t sum(int x0, int y0, int x1, int y1) const {  // inclusive corners, inside
        return I[(size_t)(y1 + 1) * (W + 1) + x1 + 1] - I[(size_t)y0 * (W + 1) + x1 + 1] -
               I[(size_t)(y1 + 1) * (W + 1) + x0] + I[(size_t)y0 * (W + 1) + x0];
    }
};

// EvalSim SSimType_SignedProduct (BlockMatcherAW1.cu:209-218 with scale
// 255, BlockMatcher1.cu:201-210 with scale 127): the signed product of the
// two values mapped to [-1, 1], times scale, truncated.
inline int signed_product(int a, int b, float scale) {
    float f1 = 2.0f * (float(a) / 255.0f - 0.5f);
    const float f2 = 2.0f * (float(b) / 255.0f - 0.5f);
    f1 *= f2;
    f1 = f1 * scale;
    return int(f1);
}

// SimValueToFloat (BlockMatcherAW1.cu:155-158): percent of the maximum
// per-pixel similarity.
inline float sim_to_float(int v, int n) { return (float(v) / float(n)) * (100.0f / float(255)); }
// SimFloatToInteger (BlockMatcherAW1.cu:172-176) into an unsigned 16-bit channel.
inline uint16_t sim_to_u16(float f) {
    float t = (f / 100.0f + 1.0f) / 2.0f;
    t = std::min(std::max(t, 0.0f), 1.0f);
    return uint16_t(t * float(65535));
}

struct SimStore {  // SSimStore (BlockMatcherNCC.cu:115-131, BlockMatcherAW1.cu:118-133)
    int prev2, prev, max, next, next2, last;
};

// One step of the argmax scan (EvalSim, BlockMatcherNCC.cu:296-329; EvalSimAW,
// BlockMatcherAW1.cu:272-307; BlockMatcher1.cu:262-300).
inline void sim_update(SimStore& s, uint16_t& disp, int v, int d) {
    if (disp > kLast) return;
    const int code = d + kFirst;
    const bool above = v > s.max;
    const bool jb = !above && int(disp) + 1 == code;
    const bool j2b = !above && int(disp) + 2 == code;
    if (above) {
        s.prev2 = s.prev;
        s.prev = s.last;
        s.max = v;
        s.next = v;
        s.next2 = v;
        disp = uint16_t(code);
    }
    if (jb) s.next = v;
    if (j2b) s.next2 = v;
    s.last = v;
}

struct MinRange {  // ushort4 (x = minimum, y = before, z = after, w = last)
    int x, y, z, w;
};

// EvalSAD's update (BlockMatcherSAD1.cu:158-190) and AW2's UpdateDisp
// (BlockMatcherAW2.cu:143-200, which also sets z at index 0).
inline void min_update(MinRange& m, uint16_t& disp, int v, int idx, int inc, int n, float thresh, bool aw2) {
    if (aw2 ? disp > kLast : disp == kCannot) return;
    const float fmin = float(v) / float(n);
    if (idx == 0) {
        m.w = v;
        m.y = v;
        if (aw2) m.z = v;
    }
    const bool below = v < m.x && fmin < thresh;
    if (below) {
        m.y = m.w;
        m.x = v;
        m.z = v;
        disp = uint16_t(idx);
    } else if (int(disp) + inc == idx) {
        m.z = v;
    }
    m.w = v;
}

}  // namespace

extern "C" {

// method: 0 SAD1 (coarse / fine SAD, BlockMatcherSAD1.cu:279-488), 1 NCC
// (BlockMatcherNCC.cu:614-884), 2 AW1 (centre + best 2 of 4 sub-windows,
// BlockMatcherAW1.cu:657-913), 3 AW2 (centre + 2 lowest of 4 sub-window SADs,
// BlockMatcherAW2.cu:404-584), 4 BM1 (plain window, BlockMatcher1.cu:590-845).
// patch: window side (SAD1 / NCC / BM1) or sub-window side s (AW1 / AW2,
// patch 3 s). sim_type (AW1, BM1): 0 absolute difference, 1 signed product.
// dir 1: base = L, match column x - d; 0: base = R, x + d. Disparities
// dmin .. dmin + D - 1. out4: W * H * 4 uint16 (x, y, z, w).
void or_compat_match(const uint8_t* L, const uint8_t* R, int W, int H, int pitch, int method, int D, int dmin,
                     int patch, int sim_type, int dir, float grad_t, float score_t, float delta_t, uint16_t* out4) {
    const uint8_t* B = dir ? L : R;
    const uint8_t* M = dir ? R : L;
    const bool aw = method == kAw1 || method == kAw2;
    const int s = patch;                       // AW sub-window side
    const int P = aw ? 3 * s : patch;          // patch side
    const int a = P / 2, b = P - 1 - a;        // patch extent left / right of the pixel
    const int n_eff = aw ? 3 * s * s : P * P;  // BasePatchElementCount
    const size_t N = (size_t)W * H;
    auto inside = [&](int x, int y) { return x - a >= 0 && x + b < W && y - a >= 0 && y + b < H; };
    auto mcol = [&](int x, int d) { return dir ? x - d : x + d; };
    auto searchable = [&](int x, int d) { const int xm = mcol(x, d); return xm - a >= 0 && xm + b < W; };

    // ---- gradient gates -----------------------------------------------------
    std::vector<uint8_t> gated(N, 0);
    if (grad_t > 0.0f) {
        std::vector<int32_t> g(N), v(N), v2(N);
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                const int p = B[y * pitch + x];
                const int q = x + 1 < W ? B[y * pitch + x + 1] : 0;  // SafeReadFromSurf fills 0
                g[(size_t)y * W + x] = std::abs(p - q);
                v[(size_t)y * W + x] = p;
                v2[(size_t)y * W + x] = p * p;
            }
        const Box bg(g.data(), W, H), bv(v.data(), W, H), bv2(v2.data(), W, H);
#pragma omp parallel for schedule(static)
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                if (!inside(x, y)) continue;
                bool gate = false;
                if (method == kSad1 || method == kNcc) {  // SAD1.cu:226-249, NCC.cu:388-413
                    const float f = float(bg.sum(x - a, y - a, x + b, y + b)) / float(P * P);
                    gate = f < grad_t;
                } else if (method == kBm1 || method == kAw1) {  // BM1.cu:327-364, AW1.cu:331-417
                    const float fm = float(bv.sum(x - a, y - a, x + b, y + b)) / float(P * P);
                    const float fm2 = float(bv2.sum(x - a, y - a, x + b, y + b)) / float(P * P);
                    float sd = std::sqrt(std::fabs(fm2 - fm * fm));
                    if (method == kAw1) sd = float(int(sd)) / float(255) * 100.0f;  // stored as int first
                    else sd = sd / float(255) * 100.0f;
                    gate = sd < grad_t;
                } else {  // AW2: the min-variant neighbourhood over gradient sub-sums (AW2.cu:216-247)
                    auto sub = [&](int cx, int cy) {
                        return int(bg.sum(cx - s / 2, cy - s / 2, cx + s / 2, cy + s / 2));
                    };
                    int e[4] = {sub(x, y - s), sub(x - s, y), sub(x, y + s), sub(x + s, y)};
                    std::sort(e, e + 4);
                    const float f = float(sub(x, y) + e[0] + e[1]) / float(n_eff);
                    gate = f < grad_t;
                }
                gated[(size_t)y * W + x] = gate ? 1 : 0;
            }
    }

    // ---- per-disparity score planes -------------------------------------------
    // NCC statistics (EvalMsd, NCC.cu:339-373; EvalSim, NCC.cu:196-236)
    std::vector<float> bmean(N), bstd(N);
    std::vector<int32_t> msum(N, 0), msum2(N, 0);
    if (method == kNcc) {
        std::vector<int32_t> v(N), v2(N), w(N), w2(N);
        for (size_t i = 0; i < N; ++i) {
            const int p = B[(i / W) * pitch + i % W], q = M[(i / W) * pitch + i % W];
            v[i] = p; v2[i] = p * p; w[i] = q; w2[i] = q * q;
        }
        const Box bv(v.data(), W, H), bv2(v2.data(), W, H), bw(w.data(), W, H), bw2(w2.data(), W, H);
        for (int y = a; y + b < H; ++y)
            for (int x = a; x + b < W; ++x) {
                const size_t o = (size_t)y * W + x;
                const float fMean = float(bv.sum(x - a, y - a, x + b, y + b)) / float(P * P);
                const float fMean2 = float(bv2.sum(x - a, y - a, x + b, y + b)) / float(P * P);
                bmean[o] = fMean;
                bstd[o] = std::sqrt(fMean2 - fMean * fMean);
                msum[o] = int32_t(bw.sum(x - a, y - a, x + b, y + b));
                msum2[o] = int32_t(bw2.sum(x - a, y - a, x + b, y + b));
            }
    }
    // score of every pixel at disparity d (valid where pixel and d are)
    auto plane = [&](int d, std::vector<int32_t>& sc) {
        std::vector<int32_t> e(N, 0);
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                const int xm = mcol(x, d);
                if (xm < 0 || xm >= W) continue;
                const int p = B[y * pitch + x], q = M[y * pitch + xm];
                int v = 0;
                switch (method) {
                    case kSad1: case kAw2: v = std::abs(p - q); break;
                    case kNcc: v = p * q; break;
                    case kAw1: v = sim_type ? int(int16_t(signed_product(p, q, 255.0f))) : 255 - std::abs(p - q); break;
                    case kBm1: v = sim_type ? signed_product(p, q, 127.0f) : (255 - std::abs(p - q)) >> 1; break;
                }
                e[(size_t)y * W + x] = v;
            }
        const Box be(e.data(), W, H);
#pragma omp parallel for schedule(static)
        for (int y = a; y < H - b; ++y)
            for (int x = a; x < W - b; ++x) {
                const size_t o = (size_t)y * W + x;
                if (!searchable(x, d)) continue;
                if (!aw) {
                    const int64_t S = be.sum(x - a, y - a, x + b, y + b);
                    if (method != kNcc) {
                        sc[o] = int32_t(S);
                        continue;
                    }
                    // NCC quantised to uint8 (NCC.cu:218-271)
                    const float fCrossMean = float(S) / float(P * P);
                    const float fTestMean = float(msum[(size_t)y * W + mcol(x, d)]) / float(P * P);
                    const float fTestMean2 = float(msum2[(size_t)y * W + mcol(x, d)]) / float(P * P);
                    const float fTestStd = std::sqrt(fTestMean2 - fTestMean * fTestMean);
                    const float fNorm = bstd[o] * fTestStd;
                    float fNcc;
                    if (fNorm < 1.0f) fNcc = 0.0f;
                    else fNcc = (fCrossMean - bmean[o] * fTestMean) / fNorm;
                    fNcc = fNcc > 0.0f ? fNcc : 0.0f;  // max(0, fNcc); NaN -> 0
                    const float f = std::min(255.0f, fNcc * 255.0f);
                    sc[o] = int32_t(uint8_t(f));
                } else {  // AW sub-window neighbourhoods (AdaptWnd_W32H16.h:240-285, AdaptWnd3D.h:244-300)
                    auto sub = [&](int cx, int cy) {
                        return int(be.sum(cx - s / 2, cy - s / 2, cx + s / 2, cy + s / 2));
                    };
                    int e4[4] = {sub(x, y - s), sub(x - s, y), sub(x, y + s), sub(x + s, y)};
                    std::sort(e4, e4 + 4);
                    sc[o] = method == kAw1 ? sub(x, y) + e4[3] + e4[2] : sub(x, y) + e4[0] + e4[1];
                }
            }
    };

    // ---- scans --------------------------------------------------------------
    std::vector<uint16_t> disp(N, kUnknown);
    for (size_t i = 0; i < N; ++i) if (gated[i]) disp[i] = kCannot;
    std::vector<int32_t> sc(N, 0);
    if (method == kNcc || method == kAw1 || method == kBm1) {
        std::vector<SimStore> st(N, SimStore{0, 0, method == kNcc ? 0 : -32767, 0, 0, 0});
        for (int d = dmin; d < dmin + D; ++d) {  // ascending (NCC.cu:789-795)
            plane(d, sc);
            for (int y = a; y < H - b; ++y)
                for (int x = a; x < W - b; ++x)
                    if (searchable(x, d)) {
                        const size_t o = (size_t)y * W + x;
                        sim_update(st[o], disp[o], method == kNcc ? sc[o] : int(int16_t(sc[o])), d);
                    }
        }
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                const size_t o = (size_t)y * W + x;
                uint16_t* px = out4 + 4 * o;
                if (!inside(x, y)) { px[0] = kCannot; px[1] = px[2] = px[3] = 0; continue; }
                const uint16_t c = disp[o];
                if (c > kLast || c == kUnknown) { px[0] = c; px[1] = px[2] = px[3] = 0; continue; }
                const SimStore& q = st[o];
                const int dw = c - kFirst;
                const bool sat = dw <= dmin + 1 || dw >= dmin + D - 1;  // First + Min + 1, First + Max - 1
                if (method == kNcc) {  // WriteDisparity, NCC.cu:520-575
                    const float fNccMax = float(q.max) / float(255);
                    const int d1 = std::max(std::abs(q.prev - q.max), std::abs(q.prev2 - q.max));
                    const int d2 = std::max(std::abs(q.next - q.max), std::abs(q.next2 - q.max));
                    uint16_t id;
                    if (fNccMax >= score_t) id = sat ? kSaturated : (d1 >= int(delta_t) && d2 >= int(delta_t) ? c : kNotSpecific);
                    else id = kNotFound;
                    px[0] = id; px[1] = uint16_t(q.max); px[2] = uint16_t(d1); px[3] = uint16_t(d2);
                } else {  // WriteDisparity, AW1.cu:533-635, BM1.cu:466-565
                    const float fMax = sim_to_float(q.max, n_eff);
                    const float fPrev2 = sim_to_float(q.prev2, n_eff), fPrev = sim_to_float(q.prev, n_eff);
                    const float fNext = sim_to_float(q.next, n_eff), fNext2 = sim_to_float(q.next2, n_eff);
                    const float fdp = std::max(std::fabs(fPrev - fMax), std::fabs(fPrev2 - fMax));
                    const float fdn = std::max(std::fabs(fNext - fMax), std::fabs(fNext2 - fMax));
                    const bool specific = fdp >= delta_t && fdn >= delta_t;
                    uint16_t id;
                    if (fMax >= score_t) id = sat ? kSaturated : (specific ? c : kNotSpecific);
                    else id = kNotFound;
                    px[0] = id; px[1] = sim_to_u16(fMax); px[2] = sim_to_u16(fdp); px[3] = sim_to_u16(fdn);
                }
            }
        return;
    }
    // SAD1 / AW2: index idx from the largest disparity (SAD1.cu:389-434, AW2.cu:539)
    std::vector<MinRange> mr(N, MinRange{0xFFFF, 0, 0, 0});
    const bool aw2 = method == kAw2;
    auto dof = [&](int idx) { return dmin + D - 1 - idx; };
    auto pass = [&](int idx, int inc, bool fine) {
        const int d = dof(idx);
        plane(d, sc);
        for (int y = a; y < H - b; ++y)
            for (int x = a; x < W - b; ++x) {
                if (!searchable(x, d)) continue;
                const size_t o = (size_t)y * W + x;
                if (fine && !(idx + 4 >= int(disp[o]) && idx <= int(disp[o]) + 4)) continue;
                min_update(mr[o], disp[o], sc[o], idx, inc, n_eff, score_t, aw2);
            }
    };
    if (aw2) {
        for (int idx = 0; idx < D; ++idx) pass(idx, 1, false);
    } else {
        for (int idx = 0; idx < D; idx += 4) pass(idx, 4, false);  // coarse
        for (int idx = 0; idx < D; ++idx) pass(idx, 1, true);      // fine
    }
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const size_t o = (size_t)y * W + x;
            uint16_t* px = out4 + 4 * o;
            if (!inside(x, y)) { px[0] = kCannot; px[1] = px[2] = px[3] = 0; continue; }
            const uint16_t c = disp[o];
            if (c > kLast) { px[0] = c; px[1] = px[2] = px[3] = 0; continue; }
            const MinRange& m = mr[o];
            const float fmin = float(m.x) / float(n_eff);
            const int d1 = std::abs(m.y - m.x), d2 = std::abs(m.z - m.x);
            const uint16_t y1 = uint16_t(m.x / n_eff);
            // the index compares against First-based bounds (SAD1.cu:459, AW2.cu:356)
            const bool sat = aw2 ? (c <= kFirst + 4 || c >= kFirst + D - 4) : (c <= kFirst + 1 || c >= kFirst + D - 1);
            const bool spec = aw2 ? (d1 >= int(delta_t) && d2 >= int(delta_t)) : (d1 > int(delta_t) && d2 > int(delta_t));
            uint16_t id;
            if (fmin < score_t) id = (spec && !sat) ? uint16_t(kFirst + dof(c)) : (sat ? kSaturated : kNotSpecific);
            else id = kNotFound;
            px[0] = id; px[1] = y1; px[2] = uint16_t(d1); px[3] = uint16_t(d2);
        }
}

// The gradient gate on its own, for the plain matchers' maps (gate.cu):
// kind 0 = mean |I(x) - I(x+1)| over the P x P patch (SAD1.cu:226-249,
// NCC.cu:388-413), 1 = standard deviation truncated to an integer, in
// percent of 255 (AW1.cu:331-417). mask[y W + x] = 1 where the pixel's patch
// is inside the image and the statistic is below thresh.
void or_gate_mask(const uint8_t* img, int W, int H, int pitch, int kind, int P, float thresh, uint8_t* mask) {
    const int a = P / 2, b = P - 1 - a;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            uint8_t g = 0;
            if (x - a >= 0 && x + b < W && y - a >= 0 && y + b < H) {
                if (kind == 0) {
                    int s = 0;
                    for (int r = y - a; r <= y + b; ++r)
                        for (int c = x - a; c <= x + b; ++c)
                            s += std::abs(int(img[r * pitch + c]) - int(c + 1 < W ? img[r * pitch + c + 1] : 0));
                    g = float(s) / float(P * P) < thresh;
                } else {
                    int s = 0, q = 0;
                    for (int r = y - a; r <= y + b; ++r)
                        for (int c = x - a; c <= x + b; ++c) {
                            const int v = img[r * pitch + c];
                            s += v;
                            q += v * v;
                        }
                    const float fm = float(s) / float(P * P), fm2 = float(q) / float(P * P);
                    const float sd = std::sqrt(std::fabs(fm2 - fm * fm));
                    g = float(int(sd)) / float(255) * 100.0f < thresh;
                }
            }
            mask[(size_t)y * W + x] = g;
        }
}

}  // extern "C"
