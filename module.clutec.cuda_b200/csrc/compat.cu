// compat.cu — the reference matchers' own output: BlockMatcherSAD1, NCC, AW1,
// AW2 and BlockMatcher1 with their 4 x uint16 TPixelEx pixel
//   x = disparity + EDisparityId::First, or Saturated / NotFound /
//       NotSpecific / CannotEvaluate / Unknown,
//   y = the winning score (SAD / N, uint8-quantised NCC, or the AW / BM
//       similarity as a 16-bit percentage),
//   z, w = the specificity channels: how far the scores next to the winner
//       fall from it, as the reference's sequential scan records them,
// the gradient gates (fGradThresh -> CannotEvaluate), the score thresholds
// (fSadThresh / fNccThresh / fSimThresh -> NotFound) and the minimum-delta
// thresholds (-> NotSpecific).
//
// Those channels come from a scan over the disparities in the reference's
// order (NCC, AW1, BM1: ascending from xDispConfig.Min(); SAD1, AW2: from the
// largest disparity down, SAD1 first in steps of 4 and then finely around
// its winner), so here one thread owns one pixel and walks the disparities
// in that order, keeping the reference's scan state in registers
// (SSimStore, BlockMatcherNCC.cu:115-131; SAD1's ushort4 min range,
// BlockMatcherSAD1.cu:158-190). A CTA owns a 32 x 8 pixel tile: its base
// region and the match strip every disparity of the scan reads are staged in
// shared memory once; per disparity the CTA writes the per-pixel similarity
// of the region into shared memory and forms the window sums in two
// separable passes (vertical, then horizontal; for the adaptive windows
// first the sub-window sums, then the centre + best / lowest 2 of 4
// neighbourhood of Kernel.Algo.AdaptWnd_W32H16.h:240-285 and
// Kernel.Algo.AdaptWnd3D.h:244-300).
//
// Pixels whose patch leaves the image get (CannotEvaluate, 0, 0, 0) (the
// reference leaves them unwritten); a disparity is searched iff the matched
// patch is inside the image. Float steps use IEEE-rounded intrinsics in the
// reference's operation order, without contraction, so results are
// bit-exact against the CPU restatement.
#include "ct_internal.h"
#include "ct_device.cuh"

namespace ct {
namespace compat {

constexpr int kTX = 32, kTY = 8, kNT = kTX * kTY;
constexpr int kPMax = 16;                  // largest patch side (SAD1 Patch_16x16)
constexpr int kRW = kTX + kPMax;           // staged base columns (one extra for the gradient)
constexpr int kRH = kTY + kPMax - 1;       // staged rows
constexpr int kMW = kTX + kPMax - 1 + 255; // staged match columns (region + D - 1)
constexpr int kSubMax = 5;                 // AW sub-window side (Patch_15x15)
// scan steps whose window sums share one round of CTA barriers (AW, with
// its sub-window planes, 2; the plain windows 4)
__host__ __device__ constexpr int steps_per_round(bool aw) { return aw ? 2 : 4; }

enum Method { kSad1 = CT_COMPAT_SAD1, kNcc = CT_COMPAT_NCC, kAw1 = CT_COMPAT_AW1, kAw2 = CT_COMPAT_AW2,
              kBm1 = CT_COMPAT_BM1 };

struct Args {
    int W, H, D, dmin, P, s, sim_type, dir;
    float grad_t, score_t, delta_t;
    const uint8_t* B;  // base image
    const uint8_t* M;  // match image
    size_t pb, pm;
    const float* mMean;  // NCC: the match image's patch mean and standard deviation (W * H,
    const float* mStd;   // EvalMsd's FP32 steps, BlockMatcherNCC.cu:222-230)
    void* out;
    size_t out_pitch;
    int out_type;
};

__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float i2f(int v) { return __int2float_rn(v); }

// RN(x / d) for an integer-valued x (|x| <= 2^24) and a positive integer
// divisor d, given zd = RN(1 / d): one multiply and the remainder correction
// of P. Markstein (IA-64 and Elementary Functions, 2000): q = RN(x zd);
// r = x - q d, exact through a fused multiply-add; q' = RN(q + r zd). Equal to
// the IEEE quotient for every numerator in that range and every divisor the
// kernels use (the patch element counts P^2, P = 1 .. 16, 3 s^2 for the
// adaptive windows, and 255), checked exhaustively against IEEE division
// (tests/test_compat_oracle.py). Three instructions instead of a division.
__device__ __forceinline__ float div_int(float x, float d, float zd) {
    const float q = __fmul_rn(x, zd);
    const float r = __fmaf_rn(-q, d, x);
    return __fmaf_rn(r, zd, q);
}

// EvalSim SSimType_SignedProduct (BlockMatcherAW1.cu:209-218 scale 255,
// BlockMatcher1.cu:201-210 scale 127), truncated.
// z255 = RN(1 / 255).
__device__ __forceinline__ int signed_product(int p, int q, float scale, float z255) {
    float f1 = fmul(2.0f, fsub(div_int(i2f(p), 255.0f, z255), 0.5f));
    const float f2 = fmul(2.0f, fsub(div_int(i2f(q), 255.0f, z255), 0.5f));
    f1 = fmul(f1, f2);
    f1 = fmul(f1, scale);
    return __float2int_rz(f1);
}

// SimValueToFloat / SimFloatToInteger (BlockMatcherAW1.cu:155-176).
__device__ __forceinline__ float sim_to_float(int v, int n) {
    return fmul(fdiv(i2f(v), i2f(n)), fdiv(100.0f, 255.0f));
}
__device__ __forceinline__ uint16_t sim_to_u16(float f) {
    float t = fdiv(fadd(fdiv(f, 100.0f), 1.0f), 2.0f);
    t = fminf(fmaxf(t, 0.0f), 1.0f);
    return uint16_t(__float2uint_rz(fmul(t, 65535.0f)));
}

__device__ __forceinline__ void store4(const Args& a, int x, int y, uint16_t c0, uint16_t c1, uint16_t c2,
                                       uint16_t c3) {
    char* row = static_cast<char*>(a.out) + (size_t)y * a.out_pitch;
    if (a.out_type == CT_PIX_U16X4)
        reinterpret_cast<ushort4*>(row)[x] = make_ushort4(c0, c1, c2, c3);
    else
        reinterpret_cast<uint16_t*>(row)[x] = c0;
}

// PC: the patch side (sub-window side for AW1 / AW2) as a compile-time
// constant, so that the window loops unroll; 0 = taken from the arguments.
template <int METHOD, int PC>
__global__ void __launch_bounds__(kNT) compat_kernel(Args a) {
    constexpr bool AW = METHOD == kAw1 || METHOD == kAw2;
    constexpr bool SIM = METHOD == kNcc || METHOD == kAw1 || METHOD == kBm1;  // argmax scan
    __shared__ uint8_t sB[kRH][kRW + 4];
    __shared__ uint8_t sM[kRH][kMW + 1];
    constexpr bool kFillE = AW || METHOD == kBm1;  // similarity staged once per step (AW; BM1's signed product)
    constexpr int kU = steps_per_round(AW);
    __shared__ int32_t sE[kFillE ? kU : 1][kFillE ? kRH : 1][kFillE ? kRW : 1];
    __shared__ int32_t sV[kU][AW ? kTY + 2 * kSubMax : kTY][kRW];
    __shared__ int32_t sH[AW ? 1 : kU][AW ? 1 : kTY][AW ? 1 : kTX];
    __shared__ int32_t sS[AW ? kU : 1][AW ? kTY + 2 * kSubMax : 1][AW ? kTX + 2 * kSubMax : 1];

    const int tid = threadIdx.x, tx = tid % kTX, ty = tid / kTX;
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
    const int x = x0 + tx, y = y0 + ty;
    constexpr bool AWm = METHOD == kAw1 || METHOD == kAw2;
    const int P = PC ? (AWm ? 3 * PC : PC) : a.P, s = PC ? (AWm ? PC : 0) : a.s, pa = P / 2, pb = P - 1 - pa;
    const int RWc = kTX + P - 1, RHc = kTY + P - 1;
    const int rx0 = x0 - pa, ry0 = y0 - pa;
    const int dmax = a.dmin + a.D - 1;
    const int mx0 = a.dir ? rx0 - dmax : rx0 + a.dmin;  // first staged match column
    const int MWc = RWc + a.D - 1;

    // stage the base region (one extra column for the gradient) and the match strip
    for (int i = tid; i < RHc * (RWc + 1); i += kNT) {
        const int r = i / (RWc + 1), c = i % (RWc + 1);
        const int xx = rx0 + c, yy = ry0 + r;
        sB[r][c] = (xx >= 0 && xx < a.W && yy >= 0 && yy < a.H) ? a.B[(size_t)yy * a.pb + xx] : 0;
    }
    for (int i = tid; i < RHc * MWc; i += kNT) {
        const int r = i / MWc, c = i % MWc;
        const int xx = mx0 + c, yy = ry0 + r;
        sM[r][c] = (xx >= 0 && xx < a.W && yy >= 0 && yy < a.H) ? a.M[(size_t)yy * a.pm + xx] : 0;
    }
    __syncthreads();

    const bool valid = x - pa >= 0 && x + pb < a.W && y - pa >= 0 && y + pb < a.H;
    const int n_eff = AW ? 3 * s * s : P * P;  // BasePatchElementCount
    const float f_eff = i2f(n_eff), z_eff = __frcp_rn(f_eff);
    const float f_pp = i2f(P * P), z_pp = __frcp_rn(f_pp);
    const float z255 = __frcp_rn(255.0f);

    // ---- gradient gate (once per pixel, directly from the staged base) ----
    bool gated = false;
    if (valid && a.grad_t > 0.0f) {
        if (METHOD == kSad1 || METHOD == kNcc) {  // mean |I(x) - I(x+1)| (SAD1.cu:226-249, NCC.cu:388-413)
            int g = 0;
            for (int r = 0; r < P; ++r)
                for (int c = 0; c < P; ++c) g += abs(int(sB[ty + r][tx + c]) - int(sB[ty + r][tx + c + 1]));
            gated = fdiv(i2f(g), i2f(P * P)) < a.grad_t;
        } else if (METHOD == kBm1 || METHOD == kAw1) {  // std. dev. in % (BM1.cu:327-364, AW1.cu:331-417)
            int sm = 0, sq = 0;
            for (int r = 0; r < P; ++r)
                for (int c = 0; c < P; ++c) {
                    const int v = sB[ty + r][tx + c];
                    sm += v;
                    sq += v * v;
                }
            const float fm = fdiv(i2f(sm), i2f(P * P)), fm2 = fdiv(i2f(sq), i2f(P * P));
            float sd = __fsqrt_rn(fabsf(fsub(fm2, fmul(fm, fm))));
            if (METHOD == kAw1) sd = fmul(fdiv(i2f(__float2int_rz(sd)), 255.0f), 100.0f);  // stored as int first
            else sd = fmul(fdiv(sd, 255.0f), 100.0f);
            gated = sd < a.grad_t;
        } else {  // AW2: centre + 2 lowest of 4 gradient sub-sums (AW2.cu:216-247)
            auto sub = [&](int cx, int cy) {  // sub-window centred at region (cx, cy)
                int g = 0;
                for (int r = -s / 2; r <= s / 2; ++r)
                    for (int c = -s / 2; c <= s / 2; ++c)
                        g += abs(int(sB[cy + r][cx + c]) - int(sB[cy + r][cx + c + 1]));
                return g;
            };
            const int cx = tx + pa, cy = ty + pa;
            const int e1 = sub(cx - s, cy), e2 = sub(cx, cy + s), e3 = sub(cx + s, cy);
            int m1 = sub(cx, cy - s), m2 = 0x7FFFFFFF;  // OrderedInsert (min): the two smallest
            m2 = min(m2, max(m1, e1)); m1 = min(m1, e1);
            m2 = min(m2, max(m1, e2)); m1 = min(m1, e2);
            m2 = min(m2, max(m1, e3)); m1 = min(m1, e3);
            gated = fdiv(i2f(sub(cx, cy) + m1 + m2), i2f(n_eff)) < a.grad_t;
        }
    }

    // ---- NCC base statistics (EvalMsd, NCC.cu:339-373) ----
    float bMean = 0.f, bStd = 0.f;
    if (METHOD == kNcc && valid) {
        int sm = 0, sq = 0;
        for (int r = 0; r < P; ++r)
            for (int c = 0; c < P; ++c) {
                const int v = sB[ty + r][tx + c];
                sm += v;
                sq += v * v;
            }
        bMean = fdiv(i2f(sm), i2f(P * P));
        bStd = __fsqrt_rn(fsub(fdiv(i2f(sq), i2f(P * P)), fmul(bMean, bMean)));
    }

    // ---- scan state ----
    uint16_t disp = gated ? uint16_t(CT_DISP_CANNOT_EVALUATE) : uint16_t(CT_DISP_UNKNOWN);
    int sPrev2 = 0, sPrev = 0, sMax = METHOD == kNcc ? 0 : -32767, sNext = 0, sNext2 = 0, sLast = 0;  // SIM
    int mX = 0xFFFF, mY = 0, mZ = 0, mW = 0;                                                        // min range
    // largest searchable disparity for this pixel
    const int dlim = a.dir ? x - pa : a.W - 1 - pb - x;

    const int nsteps = METHOD == kSad1 ? (a.D + 3) / 4 + a.D : a.D;
    // scan step k: index idx (disparity d), its increment and whether it is
    // SAD1's fine pass; the staged match column of region column 0
    struct Step {
        int idx, inc, d, moff;
        bool fine;
    };
    auto step_of = [&](int k) {
        Step st;
        st.inc = 1;
        st.fine = false;
        if (METHOD == kSad1) {
            const int nc = (a.D + 3) / 4;
            if (k < nc) { st.idx = 4 * k; st.inc = 4; }
            else { st.idx = k - nc; st.fine = true; }
        } else {
            st.idx = k;
        }
        st.d = SIM ? a.dmin + st.idx : dmax - st.idx;
        st.moff = a.dir ? dmax - st.d : st.d - a.dmin;
        return st;
    };
    for (int k0 = 0; k0 < nsteps; k0 += kU) {
        const int nu = min(kU, nsteps - k0);
        // per-pixel similarity at a round step's disparity (staged region row r, column c)
        auto sim = [&](int r, int c, int moff) {
            const int p = sB[r][c], q = sM[r][c + moff];
            if (METHOD == kSad1 || METHOD == kAw2) return abs(p - q);
            if (METHOD == kNcc) return p * q;
            if (METHOD == kAw1) return a.sim_type ? signed_product(p, q, 255.0f, z255) : 255 - abs(p - q);
            return a.sim_type ? signed_product(p, q, 127.0f, z255) : (255 - abs(p - q)) >> 1;
        };
        int Su[kU];
        if (!AW) {
            // Plain windows. Vertical P-row sums by running sums down each
            // staged column (one thread per step and column), the similarity
            // computed on the fly (SAD1, NCC, BM1's absolute difference) or
            // staged once (BM1's signed product, several FP32 steps); then
            // horizontal P-wide sums, 4 outputs per thread by running sums
            // along each row; then each pixel reads its own.
            const bool staged = kFillE && a.sim_type;
            if (staged) {
                for (int u = 0; u < nu; ++u) {
                    const int moff = step_of(k0 + u).moff;
                    for (int r = ty; r < RHc; r += kTY)
                    for (int c = tx; c < RWc; c += kTX) sE[u][r][c] = sim(r, c, moff);
                }
                __syncthreads();
            }
            for (int i = tid; i < nu * RWc; i += kNT) {
                const int u = i / RWc, c = i - u * RWc;
                const int moff = step_of(k0 + u).moff;
                auto e = [&](int r) {  // (sE has one element unless kFillE)
                    return staged ? sE[kFillE ? u : 0][kFillE ? r : 0][kFillE ? c : 0] : sim(r, c, moff);
                };
                int v = 0;
                for (int r = 0; r < P; ++r) v += e(r);
                sV[u][0][c] = v;
#pragma unroll
                for (int r = 1; r < kTY; ++r) {
                    v += e(r + P - 1) - e(r - 1);
                    sV[u][r][c] = v;
                }
            }
            __syncthreads();
            for (int i = tid; i < nu * kTY * (kTX / 4); i += kNT) {
                const int u = i / (kTY * (kTX / 4)), j = i - u * (kTY * (kTX / 4));
                const int r = j / (kTX / 4), c0 = 4 * (j % (kTX / 4));
                int v = 0;
                for (int q = 0; q < P; ++q) v += sV[u][r][c0 + q];
                sH[u][r][c0] = v;
#pragma unroll
                for (int k = 1; k < 4; ++k) {
                    v += sV[u][r][c0 + k + P - 1] - sV[u][r][c0 + k - 1];
                    sH[u][r][c0 + k] = v;
                }
            }
            __syncthreads();
#pragma unroll
            for (int u = 0; u < kU; ++u) Su[u] = u < nu ? sH[u][ty][tx] : 0;
        } else {
            for (int u = 0; u < nu; ++u) {
                const int moff = step_of(k0 + u).moff;
                for (int r = ty; r < RHc; r += kTY)
                for (int c = tx; c < RWc; c += kTX) sE[u][r][c] = sim(r, c, moff);
            }
            __syncthreads();
            const int SR = kTY + 2 * s, SC = kTX + 2 * s;
            for (int u = 0; u < nu; ++u)
                for (int r = ty; r < SR; r += kTY)
                for (int c = tx; c < RWc; c += kTX) {
                    int t = 0;
                    for (int q = 0; q < s; ++q) t += sE[u][r + q][c];
                    sV[u][r][c] = t;
                }
            __syncthreads();
            for (int u = 0; u < nu; ++u)
                for (int r = ty; r < SR; r += kTY)
                for (int c = tx; c < SC; c += kTX) {
                    int t = 0;
                    for (int q = 0; q < s; ++q) t += sV[u][r][c + q];
                    sS[u][r][c] = t;
                }
            __syncthreads();
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                if (u >= nu) {
                    Su[u] = 0;
                    continue;
                }
                const int C = sS[u][ty + s][tx + s];
                const int e0 = sS[u][ty][tx + s], e1 = sS[u][ty + s][tx], e2 = sS[u][ty + 2 * s][tx + s],
                          e3 = sS[u][ty + s][tx + 2 * s];
                if (METHOD == kAw1) {  // OrderedInsertMax: the two largest
                    int m1 = e0, m2 = -32767;
                    m2 = max(m2, min(m1, e1)); m1 = max(m1, e1);
                    m2 = max(m2, min(m1, e2)); m1 = max(m1, e2);
                    m2 = max(m2, min(m1, e3)); m1 = max(m1, e3);
                    Su[u] = C + m1 + m2;
                } else {  // OrderedInsert (min): the two smallest
                    int m1 = e0, m2 = 0x7FFFFFFF;
                    m2 = min(m2, max(m1, e1)); m1 = min(m1, e1);
                    m2 = min(m2, max(m1, e2)); m1 = min(m1, e2);
                    m2 = min(m2, max(m1, e3)); m1 = min(m1, e3);
                    Su[u] = C + m1 + m2;
                }
            }
        }
        // the scan updates of the round's steps, in scan order
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            if (u >= nu) break;
            const Step st = step_of(k0 + u);
            const int idx = st.idx, inc = st.inc, d = st.d;
            const bool fine = st.fine;
            const int S = Su[u];
            if (valid && d <= dlim) {
                if (SIM) {
                    int v;
                    if (METHOD == kNcc) {  // uint8-quantised NCC (NCC.cu:218-271)
                        const int xm = a.dir ? x - d : x + d;
                        const size_t om = (size_t)y * a.W + xm;
                        const float fCross = div_int(i2f(S), f_pp, z_pp);
                        const float fTm = __ldg(&a.mMean[om]);
                        const float fTstd = __ldg(&a.mStd[om]);
                        const float fNorm = fmul(bStd, fTstd);
                        float fNcc = fNorm < 1.0f ? 0.0f : fdiv(fsub(fCross, fmul(bMean, fTm)), fNorm);
                        fNcc = fNcc > 0.0f ? fNcc : 0.0f;
                        v = int(__float2uint_rz(fminf(255.0f, fmul(fNcc, 255.0f))) & 0xFFu);
                    } else {
                        v = int(int16_t(S));
                    }
                    // EvalSim's bookkeeping (NCC.cu:296-329, AW1.cu:272-307, BM1.cu:262-300)
                    if (disp <= CT_DISP_LAST) {
                        const int code = d + CT_DISP_FIRST;
                        const bool above = v > sMax;
                        const bool jb = !above && int(disp) + 1 == code;
                        const bool j2b = !above && int(disp) + 2 == code;
                        if (above) {
                            sPrev2 = sPrev; sPrev = sLast; sMax = v; sNext = v; sNext2 = v;
                            disp = uint16_t(code);
                        }
                        if (jb) sNext = v;
                        if (j2b) sNext2 = v;
                        sLast = v;
                    }
                } else {
                    // SAD1 EvalSAD (SAD1.cu:158-190), AW2 UpdateDisp (AW2.cu:143-200)
                    const bool eval = !fine || (idx + 4 >= int(disp) && idx <= int(disp) + 4);
                    const bool skip = METHOD == kAw2 ? disp > CT_DISP_LAST : disp == CT_DISP_CANNOT_EVALUATE;
                    if (eval && !skip) {
                        const int v = S;
                        const float fmin = div_int(i2f(v), f_eff, z_eff);
                        if (idx == 0) {
                            mW = v; mY = v;
                            if (METHOD == kAw2) mZ = v;
                        }
                        const bool below = v < mX && fmin < a.score_t;
                        if (below) {
                            mY = mW; mX = v; mZ = v;
                            disp = uint16_t(idx);
                        } else if (int(disp) + inc == idx) {
                            mZ = v;
                        }
                        mW = v;
                    }
                }
            }
        }
        __syncthreads();  // the next round overwrites sE / sV / sS
    }

    if (x >= a.W || y >= a.H) return;
    if (!valid) {
        store4(a, x, y, CT_DISP_CANNOT_EVALUATE, 0, 0, 0);
        return;
    }
    if (SIM) {
        if (disp > CT_DISP_LAST || disp == CT_DISP_UNKNOWN) {
            store4(a, x, y, disp, 0, 0, 0);
            return;
        }
        const int dw = int(disp) - CT_DISP_FIRST;
        const bool sat = dw <= a.dmin + 1 || dw >= a.dmin + a.D - 1;
        if (METHOD == kNcc) {  // WriteDisparity (NCC.cu:520-575)
            const float fNccMax = fdiv(i2f(sMax), 255.0f);
            const int d1 = max(abs(sPrev - sMax), abs(sPrev2 - sMax));
            const int d2 = max(abs(sNext - sMax), abs(sNext2 - sMax));
            const int thr = int(a.delta_t);
            uint16_t id;
            if (fNccMax >= a.score_t) id = sat ? CT_DISP_SATURATED : (d1 >= thr && d2 >= thr ? disp : CT_DISP_NOT_SPECIFIC);
            else id = CT_DISP_NOT_FOUND;
            store4(a, x, y, id, uint16_t(sMax), uint16_t(d1), uint16_t(d2));
        } else {  // WriteDisparity (AW1.cu:533-635, BM1.cu:466-565)
            const float fMax = sim_to_float(sMax, n_eff);
            const float fp2 = sim_to_float(sPrev2, n_eff), fp = sim_to_float(sPrev, n_eff);
            const float fn = sim_to_float(sNext, n_eff), fn2 = sim_to_float(sNext2, n_eff);
            const float fdp = fmaxf(fabsf(fsub(fp, fMax)), fabsf(fsub(fp2, fMax)));
            const float fdn = fmaxf(fabsf(fsub(fn, fMax)), fabsf(fsub(fn2, fMax)));
            const bool specific = fdp >= a.delta_t && fdn >= a.delta_t;
            uint16_t id;
            if (fMax >= a.score_t) id = sat ? CT_DISP_SATURATED : (specific ? disp : CT_DISP_NOT_SPECIFIC);
            else id = CT_DISP_NOT_FOUND;
            store4(a, x, y, id, sim_to_u16(fMax), sim_to_u16(fdp), sim_to_u16(fdn));
        }
        return;
    }
    if (disp > CT_DISP_LAST) {
        store4(a, x, y, disp, 0, 0, 0);
        return;
    }
    // SAD1 / AW2 output (SAD1.cu:438-486, AW2.cu:330-370): disp holds the scan
    // index, compared against First-based bounds as the reference does
    const float fmin = fdiv(i2f(mX), i2f(n_eff));
    const int d1 = abs(mY - mX), d2 = abs(mZ - mX);
    const int c = disp;
    const bool sat = METHOD == kAw2 ? (c <= CT_DISP_FIRST + 4 || c >= CT_DISP_FIRST + a.D - 4)
                                    : (c <= CT_DISP_FIRST + 1 || c >= CT_DISP_FIRST + a.D - 1);
    const int thr = int(a.delta_t);
    const bool spec = METHOD == kAw2 ? (d1 >= thr && d2 >= thr) : (d1 > thr && d2 > thr);
    uint16_t id;
    if (fmin < a.score_t) id = (spec && !sat) ? uint16_t(CT_DISP_FIRST + dmax - c) : (sat ? CT_DISP_SATURATED : CT_DISP_NOT_SPECIFIC);
    else id = CT_DISP_NOT_FOUND;
    store4(a, x, y, id, uint16_t(mX / n_eff), uint16_t(d1), uint16_t(d2));
}

// Mean and standard deviation of every pixel's P x P patch [x - P/2,
// x - P/2 + P - 1] of the match image, in the reference's FP32 steps
// (fTestMean = S / P^2, fTestMean2 = Q / P^2, sqrt(fTestMean2 - fTestMean^2));
// 0 where the patch leaves the image (never read there).
__global__ void __launch_bounds__(kNT) box_sq_kernel(const uint8_t* img, size_t pitch, int W, int H, int P,
                                                     float* mean, float* sd) {
    // separable: the (32 + P - 1) x (8 + P - 1) region of a 32 x 8 tile,
    // row sums of P pixels (values and squares), then column sums of P rows
    __shared__ uint8_t t[kTY + kPMax - 1][kTX + kPMax];
    __shared__ int hs[kTY + kPMax - 1][kTX], hq[kTY + kPMax - 1][kTX];
    const int tx = threadIdx.x % kTX, ty = threadIdx.x / kTX;
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY, pa = P / 2;
    const int RW = kTX + P - 1, RH = kTY + P - 1;
    for (int r = ty; r < RH; r += kTY)
        for (int c = tx; c < RW; c += kTX) {
            const int yy = y0 - pa + r, xx = x0 - pa + c;
            t[r][c] = (xx >= 0 && xx < W && yy >= 0 && yy < H) ? img[(size_t)yy * pitch + xx] : 0;
        }
    __syncthreads();
    for (int r = ty; r < RH; r += kTY) {
        int sv = 0, sq = 0;
        for (int c = 0; c < P; ++c) {
            const int v = t[r][tx + c];
            sv += v;
            sq += v * v;
        }
        hs[r][tx] = sv;
        hq[r][tx] = sq;
    }
    __syncthreads();
    const int x = x0 + tx, y = y0 + ty;
    if (x >= W || y >= H) return;
    const int pb = P - 1 - pa;
    int sv = 0, sq = 0;
    if (x - pa >= 0 && x + pb < W && y - pa >= 0 && y + pb < H)
        for (int r = 0; r < P; ++r) {
            sv += hs[ty + r][tx];
            sq += hq[ty + r][tx];
        }
    const float fTm = fdiv(i2f(sv), i2f(P * P));
    const float fTm2 = fdiv(i2f(sq), i2f(P * P));
    mean[(size_t)y * W + x] = fTm;
    sd[(size_t)y * W + x] = __fsqrt_rn(fsub(fTm2, fmul(fTm, fTm)));
}

}  // namespace compat

namespace {

struct CompatHandle : ct_handle {
    CompatHandle() : ct_handle(Kind::Compat) {}
    ~CompatHandle() override {
        if (device >= 0) cudaSetDevice(device);
        cudaFree(stats);
    }
    ct_format fmt{};
    ct_compat_params par{};
    float* stats = nullptr;  // NCC: patch mean and standard deviation planes of the match image
};

}  // namespace
}  // namespace ct

using namespace ct;

extern "C" {

int ct_bm_compat_create(ct_handle** out) {
    clear_error();
    if (!out) return fail(CT_EINVAL, "null output handle pointer");
    *out = new CompatHandle();
    return CT_OK;
}

int ct_bm_compat_configure(ct_handle* hh, int32_t device, const ct_format* fmt, const ct_compat_params* p) {
    clear_error();
    auto* h = (hh && hh->kind == Kind::Compat) ? static_cast<CompatHandle*>(hh) : nullptr;
    if (!h) return fail(CT_ESTATE, "not a reference-compat matcher handle");
    if (!fmt || !p) return fail(CT_EINVAL, "null format or parameters");
    if (fmt->type != CT_PIX_U8) return fail(CT_ETYPE, "matcher input must be U8 (TPixel_Lum_UInt8)");
    if (fmt->width < 16 || fmt->height < 16 || fmt->width > 32768 || fmt->height > 32768)
        return fail(CT_EINVAL, "image size %dx%d out of range (16..32768)", fmt->width, fmt->height);
    if (p->disp_count < 1 || p->disp_count > 256) return fail(CT_EINVAL, "disp_count must be 1..256");
    if (p->disp_min < 0 || p->disp_min + p->disp_count > 0xFFEF)
        return fail(CT_EINVAL, "disp_min must be >= 0 with disp_min + disp_count <= 65519");
    if (p->sim_type != 0 && p->sim_type != 1) return fail(CT_EINVAL, "sim_type must be 0 or 1");
    if (p->sim_type && p->method != CT_COMPAT_AW1 && p->method != CT_COMPAT_BM1)
        return fail(CT_EINVAL, "the signed product is an AW1 / BlockMatcher1 similarity");
    if (p->reserved[0] || p->reserved[1] || p->reserved[2]) return fail(CT_EINVAL, "reserved fields must be 0");
    switch (p->method) {
        case CT_COMPAT_SAD1:
            if (p->patch < 3 || p->patch > 16) return fail(CT_EINVAL, "SAD1 patch must be 3..16");
            break;
        case CT_COMPAT_NCC:
            if (p->patch != 5 && p->patch != 9 && p->patch != 11)
                return fail(CT_EINVAL, "NCC patch must be 11 (Patch_11x11), 9 or 5");
            break;
        case CT_COMPAT_BM1:
            if (p->patch != 5 && p->patch != 9 && p->patch != 11 && p->patch != 15)
                return fail(CT_EINVAL, "BlockMatcher1 patch must be 5, 9, 11 or 15");
            break;
        case CT_COMPAT_AW1:
        case CT_COMPAT_AW2:
            if (p->patch != 3 && p->patch != 5)
                return fail(CT_EINVAL, "AW sub-window must be 3 (Patch_9x9) or 5 (Patch_15x15)");
            break;
        default:
            return fail(CT_EINVAL, "unknown method %d", p->method);
    }
    if (int rc = use_device(device)) return rc;
    cudaFree(h->stats);
    h->stats = nullptr;
    h->device = device;
    if (int rc = h->init_status()) return rc;
    if (p->method == CT_COMPAT_NCC &&
        cudaMalloc(&h->stats, 2 * (size_t)fmt->width * fmt->height * sizeof(float)) != cudaSuccess)
        return fail(CT_ENOMEM, "statistics scratch");
    h->fmt = *fmt;
    h->par = *p;
    h->configured = true;
    return CT_OK;
}

int ct_bm_compat_process(ct_handle* hh, const ct_image* disp, const ct_image* left, const ct_image* right,
                         ct_stream stream) {
    clear_error();
    auto* h = (hh && hh->kind == Kind::Compat) ? static_cast<CompatHandle*>(hh) : nullptr;
    if (!h) return fail(CT_ESTATE, "not a reference-compat matcher handle");
    if (!h->configured) return fail(CT_ESTATE, "process before configure");
    if (int rc = check_image(left, "left", 1u << CT_PIX_U8)) return rc;
    if (int rc = check_image(right, "right", 1u << CT_PIX_U8)) return rc;
    if (int rc = check_same_size(left, right, "left", "right")) return rc;
    if (left->width != h->fmt.width || left->height != h->fmt.height)
        return fail(CT_EFORMAT, "image size differs from the configured format");
    if (int rc = check_image(disp, "disp", (1u << CT_PIX_U16X4) | (1u << CT_PIX_U16))) return rc;
    if (int rc = check_same_size(disp, left, "disp", "left")) return rc;
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    const ct_compat_params& p = h->par;
    const bool aw = p.method == CT_COMPAT_AW1 || p.method == CT_COMPAT_AW2;
    const ct_image* B = p.left_to_right ? left : right;
    const ct_image* M = p.left_to_right ? right : left;
    compat::Args a{};
    a.W = h->fmt.width; a.H = h->fmt.height; a.D = p.disp_count; a.dmin = p.disp_min;
    a.s = aw ? p.patch : 0;
    a.P = aw ? 3 * p.patch : p.patch;
    a.sim_type = p.sim_type;
    a.dir = p.left_to_right ? 1 : 0;
    a.grad_t = p.grad_thresh; a.score_t = p.score_thresh; a.delta_t = p.min_delta_thresh;
    a.B = static_cast<const uint8_t*>(B->ptr); a.pb = B->pitch_bytes;
    a.M = static_cast<const uint8_t*>(M->ptr); a.pm = M->pitch_bytes;
    a.out = disp->ptr; a.out_pitch = disp->pitch_bytes; a.out_type = disp->type;
    if (p.method == CT_COMPAT_NCC) {
        const size_t N = (size_t)a.W * a.H;
        a.mMean = h->stats;
        a.mStd = h->stats + N;
        compat::box_sq_kernel<<<dim3((a.W + compat::kTX - 1) / compat::kTX, (a.H + compat::kTY - 1) / compat::kTY),
                                compat::kNT, 0, s>>>(a.M, a.pm, a.W, a.H, a.P, h->stats, h->stats + N);
        CT_LAUNCH_CHECK();
    }
    const dim3 grid((a.W + compat::kTX - 1) / compat::kTX, (a.H + compat::kTY - 1) / compat::kTY);
#define CT_COMPAT_LAUNCH(M, PC) compat::compat_kernel<M, PC><<<grid, compat::kNT, 0, s>>>(a)
    const int pc = p.patch;
    switch (p.method) {
        case CT_COMPAT_SAD1:
            if (pc == 16) CT_COMPAT_LAUNCH(CT_COMPAT_SAD1, 16);
            else CT_COMPAT_LAUNCH(CT_COMPAT_SAD1, 0);
            break;
        case CT_COMPAT_NCC:
            if (pc == 11) CT_COMPAT_LAUNCH(CT_COMPAT_NCC, 11);
            else if (pc == 9) CT_COMPAT_LAUNCH(CT_COMPAT_NCC, 9);
            else CT_COMPAT_LAUNCH(CT_COMPAT_NCC, 5);
            break;
        case CT_COMPAT_AW1:
            if (pc == 3) CT_COMPAT_LAUNCH(CT_COMPAT_AW1, 3);
            else CT_COMPAT_LAUNCH(CT_COMPAT_AW1, 5);
            break;
        case CT_COMPAT_AW2:
            if (pc == 3) CT_COMPAT_LAUNCH(CT_COMPAT_AW2, 3);
            else CT_COMPAT_LAUNCH(CT_COMPAT_AW2, 5);
            break;
        default:
            if (pc == 5) CT_COMPAT_LAUNCH(CT_COMPAT_BM1, 5);
            else if (pc == 9) CT_COMPAT_LAUNCH(CT_COMPAT_BM1, 9);
            else if (pc == 11) CT_COMPAT_LAUNCH(CT_COMPAT_BM1, 11);
            else CT_COMPAT_LAUNCH(CT_COMPAT_BM1, 15);
            break;
    }
#undef CT_COMPAT_LAUNCH
    CT_LAUNCH_CHECK();
    return CT_OK;
}

}  // extern "C"
