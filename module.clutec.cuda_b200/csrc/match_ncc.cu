// match_ncc.cu — BlockMatcherNCC::CDriver with an unquantised FP32 score.
//
// The reference forms NCC from integer window sums and normalises in FP32
// through means and standard deviations (BlockMatcherNCC.cu:182-262), which
// cancels badly. Here every window sum is an exact int32 (11x11 x 255^2 fits)
// and only the last step is FP32, with IEEE-rounded operations:
//   num = n Sxy - Sx Sy,  vx = n Sxx - Sx^2,  vy = n Syy - Sy^2   (exact ints)
//   ncc = 0 if vx * vy < n^4 (sigma_x sigma_y < 1, NCC.cu:255-262)
//   ncc = float(num) / sqrt(float(vx) * float(vy)) otherwise.
// Per-pixel (Sx, vx) of both images come from a box-statistics pass; the
// matching kernel keeps vertical running sums of L(x) R(x-d) for 4 columns x
// 8 disparities per thread (same CTA decomposition as the other matchers) and
// merges the argmax through 64-bit keys (ordered score << 32 | ~d): the
// highest score wins, then the lowest d.
#include "ct_internal.h"
#include "ct_device.cuh"
#include "guide.cuh"

namespace ct {
namespace ncc {

constexpr int kCPT = 4, kTWV = 128, kDPW = 8, kNW = 8, kNT = kNW * 32, kDPC = kDPW * kNW;
constexpr int kBW = kTWV + 16, kMWs = kTWV + kDPC + 16;

__host__ __device__ constexpr int two_of(int R) { return kTWV - 2 * R; }
__host__ __device__ constexpr size_t strip_bytes(int th, int R) {
    return (size_t(kBW) * (th + 2 * R) + 127) / 128 * 128 + (size_t(kMWs) * (th + 2 * R) + 127) / 128 * 128;
}
__host__ __device__ constexpr size_t smem_bytes(int th, int R) {
    return strip_bytes(th, R) + size_t(th) * two_of(R) * 8 + 16;
}

// Box sum S and n*Q - S^2 of every pixel (the window zero-padded outside
// the image; the matchers read them only where it is inside) for both views
// in one launch (blockIdx.z: 0 the left view, which also gets T, 1 the right
// view), and the zero-score threshold of the left view: the smallest vy with
// V * vy >= n^4, i.e. ceil(n^4 / V) (INT_MAX when V = 0), so that the
// matcher's test sigma_x sigma_y >= 1 is one 32-bit compare vy >= T.
// Separable: a CTA stages a (32 + 2R) x (64 + 2R) tile (aligned words), sums every staged
// row horizontally (running sums over 4 columns a thread) into shared
// memory, then each thread runs a vertical sum down 8 rows of its column.
template <int R>
__global__ void __launch_bounds__(256) box_stats_kernel(const uint8_t* imgL, size_t pitchL, const uint8_t* imgR,
                                                        size_t pitchR, int W, int H, int32_t* SL, int32_t* VL,
                                                        int32_t* TL, int32_t* SR, int32_t* VR) {
    constexpr int TX = 32, TY = 64, K = 2 * R + 1, SH = TY + 2 * R;
    // staged rows: 12 aligned words from x0 - 8 (x0 - R .. x0 + 31 + R at
    // byte offset 8 - R); image pointers and pitches are 16-byte aligned, so
    // a word starting inside a row lies inside the pitch
    constexpr int NWd = 12;
    static_assert(R <= 8 && TX + 2 * R + (8 - R) <= 4 * NWd, "staged words cover the tile");
    __shared__ uint32_t tw[SH][NWd];
    __shared__ int hs[SH][TX], hq[SH][TX];
    const bool right = blockIdx.z != 0;
    const uint8_t* img = right ? imgR : imgL;
    const size_t pitch = right ? pitchR : pitchL;
    int32_t* S = right ? SR : SL;
    int32_t* V = right ? VR : VL;
    int32_t* T = right ? nullptr : TL;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int tid = threadIdx.y * TX + threadIdx.x;
    for (int i = tid; i < SH * NWd; i += TX * 8) {
        const int r = i / NWd, wc = i % NWd;
        const int yy = y0 - R + r, xw = x0 - 8 + 4 * wc;
        uint32_t v = 0;
        if (yy >= 0 && yy < H && xw >= 0 && xw < W) {
            v = *reinterpret_cast<const uint32_t*>(img + (size_t)yy * pitch + xw);
            if (xw + 4 > W) v &= 0xFFFFFFFFu >> (8 * (xw + 4 - W));  // bytes at x >= W read 0
        }
        tw[r][wc] = v;
    }
    __syncthreads();
    for (int i = tid; i < SH * (TX / 4); i += TX * 8) {
        const int r = i / (TX / 4), c = 4 * (i % (TX / 4));
        int v[K + 3];
#pragma unroll
        for (int k = 0; k < K + 3; ++k) v[k] = reinterpret_cast<const uint8_t*>(tw[r])[8 - R + c + k];
        int s = 0, q = 0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            s += v[k];
            q += v[k] * v[k];
        }
        hs[r][c] = s;
        hq[r][c] = q;
#pragma unroll
        for (int j = 1; j < 4; ++j) {
            s += v[j + K - 1] - v[j - 1];
            q += v[j + K - 1] * v[j + K - 1] - v[j - 1] * v[j - 1];
            hs[r][c + j] = s;
            hq[r][c + j] = q;
        }
    }
    __syncthreads();
    constexpr int n = K * K;
    constexpr long long n4 = (long long)n * n * n * n;
    static_assert(n4 < 0x7FFFFFFFll, "the threshold fits in int32");
    // n^4 + V - 1 < 2^32 (V <= n^2 255^2 / 4): one 32-bit division
    static_assert(n4 + (long long)n * n * 255 * 255 / 4 < 0xFFFFFFFFll, "32-bit threshold division");
    const int x = x0 + threadIdx.x, r0 = 8 * threadIdx.y;
    int s = 0, q = 0;
#pragma unroll
    for (int dy = 0; dy < K; ++dy) {
        s += hs[r0 + dy][threadIdx.x];
        q += hq[r0 + dy][threadIdx.x];
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        if (k > 0) {
            s += hs[r0 + k + K - 1][threadIdx.x] - hs[r0 + k - 1][threadIdx.x];
            q += hq[r0 + k + K - 1][threadIdx.x] - hq[r0 + k - 1][threadIdx.x];
        }
        const int y = y0 + r0 + k;
        if (x < W && y < H) {
            const int v = n * q - s * s;
            S[(size_t)y * W + x] = s;
            V[(size_t)y * W + x] = v;
            if (T) T[(size_t)y * W + x] = v > 0 ? int32_t((uint32_t(n4) + uint32_t(v) - 1u) / uint32_t(v)) : 0x7FFFFFFF;
        }
    }
}

__device__ __forceinline__ uint32_t ordered(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unordered(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o);
}

constexpr int kGuideBlock = guide::kBlock;

struct Args {
    int W, H, D, th;
    int dmin;                // relative d matches column x - (dmin + d); maps store dmin + d
    const uint32_t* guide;   // per 16 x 16 block search range, or null (search all D)
    int guide_gw;
    const int32_t *Sx, *Vx, *Sy, *Vy;   // stats of the left / right image (W*H)
    const int32_t* Tx;                  // zero-score threshold of the left image (box_stats_kernel)
    unsigned long long* keys;          // global keys when gridDim.z > 1 (0 between calls)
    uint32_t* counters;                // gridDim.z > 1: CTAs done per (strip, column tile), 0 between calls
    void* out;
    size_t out_pitch;
    int out_type;
    float* score;
    size_t score_pitch;
    int32_t* status;
};

__device__ __forceinline__ void store_ncc(const Args& a, int x, int y, bool valid, unsigned long long key) {
    const bool ok = valid && key != 0ull;
    const uint32_t d = ok ? 0xFFFFFFFFu - uint32_t(key & 0xFFFFFFFFull) + uint32_t(a.dmin) : 0u;
    char* row = static_cast<char*>(a.out) + (size_t)y * a.out_pitch;
    if (a.out_type == CT_PIX_U8) reinterpret_cast<uint8_t*>(row)[x] = ok ? uint8_t(d) : uint8_t(0xFF);
    else reinterpret_cast<uint16_t*>(row)[x] = ok ? uint16_t(d + 1) : uint16_t(0xFFFF);
    if (a.score)
        reinterpret_cast<float*>(reinterpret_cast<char*>(a.score) + (size_t)y * a.score_pitch)[x] =
            ok ? unordered(uint32_t(key >> 32)) : 0.0f;
}

template <int R>
__global__ void __launch_bounds__(kNT, 2)
    ncc_match_kernel(const __grid_constant__ CUtensorMap tmB, const __grid_constant__ CUtensorMap tmM, Args a) {
    constexpr int TWO = two_of(R);
    constexpr int n = (2 * R + 1) * (2 * R + 1);
    extern __shared__ __align__(128) unsigned char smem[];
    const int NR = a.th + 2 * R;
    uint8_t* sB = smem;
    uint8_t* sM = smem + (size_t(kBW) * NR + 127) / 128 * 128;
    unsigned long long* sKey = reinterpret_cast<unsigned long long*>(smem + strip_bytes(a.th, R));
    uint64_t* bar = reinterpret_cast<uint64_t*>(sKey + a.th * TWO);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int xs = blockIdx.x * TWO - R;
    const int y0 = blockIdx.y * a.th;

    if (tid == 0) {
        dev::prefetch_tmap(&tmB);
        dev::prefetch_tmap(&tmM);
        dev::mbar_init(bar, 1);
        dev::fence_barrier_init();
    }
    for (int i = tid; i < a.th * TWO; i += kNT) sKey[i] = 0ull;
    // Disparity block z covers dz0 = base + z kDPC .. + kDPC - 1. Unguided,
    // base = 0. Guided, base starts at the low end (rounded down to kDPW) of
    // the union of the search ranges of the 16 x 16 blocks this tile's
    // outputs fall in, so a tile whose union is narrow needs one block; the
    // others, and the warps of a block above the union, do no matching (the
    // outputs are still written below).
    int base = 0, ulo = 0, uhi = a.D - 1;
    if (a.guide) {
        const int2 u = guide::tile_union(a.guide, a.guide_gw, xs + R, min(xs + R + TWO, a.W) - 1, y0,
                                         min(y0 + a.th, a.H) - 1, reinterpret_cast<int*>(bar + 1));
        ulo = u.x;
        uhi = min(u.y, a.D - 1);
        if (ulo <= uhi) base = ulo & ~(kDPW - 1);
    }
    const int dz0 = base + int(blockIdx.z) * kDPC;
    const int dw = dz0 + warp * kDPW;
    const bool warp_active = dw < a.D;
    const bool searches = ulo <= uhi && dw <= uhi && dw + kDPW - 1 >= ulo;
    const int ab = xs & ~15;
    const int am = (xs - a.dmin - dz0 - (kDPC - 1)) & ~15;
    __syncthreads();
    if (tid == 0) {
        dev::mbar_arrive_expect_tx(bar, uint32_t(kBW * NR + kMWs * NR));
        dev::tma_load_2d(sB, &tmB, ab, y0 - R, bar);
        dev::tma_load_2d(sM, &tmM, am, y0 - R, bar);
    }
    const bool got = dev::mbar_wait_bounded(bar, 0);
    // a strip that never arrived: report, match nothing, still take part in
    // the merge below so that the group's counter and keys stay consistent
    const bool aborted = __syncthreads_or(!got);
    if (aborted && tid == 0) dev::report(a.status, CT_ETIMEOUT);
    const int bo = xs - ab + 4 * lane;
    const int mo = (xs - a.dmin - dz0 - am) + 4 * lane - kDPW * warp - 7;

    int V[kDPW][kCPT];
#pragma unroll
    for (int j = 0; j < kDPW; ++j)
#pragma unroll
        for (int c = 0; c < kCPT; ++c) V[j][c] = 0;

    if (warp_active && searches && !aborted) {
        for (int i = 0; i < NR; ++i) {
            {
                const uint8_t* rb = sB + i * kBW + bo;
                const uint8_t* rm = sM + i * kMWs + mo;
                int b[kCPT], m[11];
#pragma unroll
                for (int c = 0; c < kCPT; ++c) b[c] = rb[c];
#pragma unroll
                for (int k = 0; k < 11; ++k) m[k] = rm[k];
                if (i >= 2 * R + 1) {
                    const uint8_t* ob = sB + (i - 2 * R - 1) * kBW + bo;
                    const uint8_t* om = sM + (i - 2 * R - 1) * kMWs + mo;
                    int bb[kCPT], mm[11];
#pragma unroll
                    for (int c = 0; c < kCPT; ++c) bb[c] = ob[c];
#pragma unroll
                    for (int k = 0; k < 11; ++k) mm[k] = om[k];
#pragma unroll
                    for (int j = 0; j < kDPW; ++j)
#pragma unroll
                        for (int c = 0; c < kCPT; ++c)
                            V[j][c] += b[c] * m[c - j + 7] - bb[c] * mm[c - j + 7];
                } else {
#pragma unroll
                    for (int j = 0; j < kDPW; ++j)
#pragma unroll
                        for (int c = 0; c < kCPT; ++c) V[j][c] += b[c] * m[c - j + 7];
                }
            }
            if (i < 2 * R) continue;
            const int oy = i - 2 * R;
            const int y = y0 + oy;
            int C[kDPW][kCPT];
#pragma unroll
            for (int j = 0; j < kDPW; ++j) {
                int win[kCPT + 2 * R];
#pragma unroll
                for (int q = 0; q < R; ++q) {
                    const int h = R - 1 - q;
                    win[q] = __shfl_up_sync(0xffffffffu, V[j][3 - (h % 4)], h / 4 + 1);
                }
#pragma unroll
                for (int c = 0; c < kCPT; ++c) win[R + c] = V[j][c];
#pragma unroll
                for (int h = 0; h < R; ++h) win[R + kCPT + h] = __shfl_down_sync(0xffffffffu, V[j][h % 4], h / 4 + 1);
                int s = 0;
#pragma unroll
                for (int q = 0; q <= 2 * R; ++q) s += win[q];
                C[j][0] = s;
#pragma unroll
                for (int c = 1; c < kCPT; ++c) { s = s + win[c + 2 * R] - win[c - 1]; C[j][c] = s; }
            }
            if (y < R || y >= a.H - R) continue;
            // right-view statistics of the 11 match columns this thread's 4
            // columns x 8 disparities read: column xs + 4 lane - dmin - dw - 7 + k
            int syk[kCPT + kDPW - 1], vyk[kCPT + kDPW - 1];
            float ryk[kCPT + kDPW - 1];  // ~1 / sqrt(vy) of those columns (estimates only)
            {
                const int cb = xs + 4 * lane - a.dmin - dw - (kDPW - 1);
                const size_t ob = (size_t)y * a.W;
#pragma unroll
                for (int k = 0; k < kCPT + kDPW - 1; ++k) {
                    const bool in = cb + k >= 0 && cb + k < a.W;
                    syk[k] = in ? __ldg(&a.Sy[ob + cb + k]) : 0;
                    vyk[k] = in ? __ldg(&a.Vy[ob + cb + k]) : 0;
                    ryk[k] = rsqrtf(__int2float_rn(vyk[k]));
                }
            }
            // The IEEE score (a divide and a square root) decides the winner.
            // Per column, disparities are ranked by the estimate
            // num * rsqrt(vy), the score times sqrt(vx) (a positive factor
            // common to the column) within a few ulp (relative 1e-6); the
            // IEEE score is evaluated for the lowest disparity whose estimate
            // lies within 2e-5 (relative) of the column's best, and then for
            // the other such near-ties in a warp-synchronous loop (rare):
            // the rest cannot win or tie. An estimate is exactly 0 if and only
            // if the score is +0 (num = 0, or sigma_x sigma_y < 1, tested as
            // vy >= Tx), so a column whose best estimate is 0 needs no IEEE
            // work. Every lane runs every step (columns without an output
            // have no candidates).
            int sxc[kCPT] = {}, tc[kCPT] = {};
            float fvxc[kCPT] = {};
            uint32_t cand[kCPT];  // per column: near-tie candidates left after the first
            unsigned long long best[kCPT];
            // v[j] of eight registers by a three-level select on the bits of j
            auto sel8 = [](int v0, int v1, int v2, int v3, int v4, int v5, int v6, int v7, int j) {
                const bool b0 = j & 1, b1 = j & 2, b2 = j & 4;
                const int a0 = b0 ? v1 : v0, a1 = b0 ? v3 : v2, a2 = b0 ? v5 : v4, a3 = b0 ? v7 : v6;
                const int c0 = b1 ? a1 : a0, c1 = b1 ? a3 : a2;
                return b2 ? c1 : c0;
            };
            // key of disparity j of column c: IEEE score << 32 | ~d
            auto exact_key = [&](int c, int j) {
#define CT_SEL_C(q) C[q][c]
#define CT_SEL_K(arr, q) arr[c - (q) + kDPW - 1]
                static_assert(kDPW == 8, "sel8 selects among 8 disparities");
                const int cq = sel8(CT_SEL_C(0), CT_SEL_C(1), CT_SEL_C(2), CT_SEL_C(3), CT_SEL_C(4), CT_SEL_C(5),
                                    CT_SEL_C(6), CT_SEL_C(7), j);
                const int sy = sel8(CT_SEL_K(syk, 0), CT_SEL_K(syk, 1), CT_SEL_K(syk, 2), CT_SEL_K(syk, 3),
                                    CT_SEL_K(syk, 4), CT_SEL_K(syk, 5), CT_SEL_K(syk, 6), CT_SEL_K(syk, 7), j);
                const int vy = sel8(CT_SEL_K(vyk, 0), CT_SEL_K(vyk, 1), CT_SEL_K(vyk, 2), CT_SEL_K(vyk, 3),
                                    CT_SEL_K(vyk, 4), CT_SEL_K(vyk, 5), CT_SEL_K(vyk, 6), CT_SEL_K(vyk, 7), j);
#undef CT_SEL_C
#undef CT_SEL_K
                const int num = n * cq - sxc[c] * sy;
                const float sc =
                    vy >= tc[c] ? __fdiv_rn(__int2float_rn(num), __fsqrt_rn(__fmul_rn(fvxc[c], __int2float_rn(vy))))
                                : 0.0f;
                return ((unsigned long long)ordered(sc) << 32) | (0xFFFFFFFFu - uint32_t(dw + j));
            };
#pragma unroll
            for (int c = 0; c < kCPT; ++c) {
                const int v = 4 * lane + c;
                const int x = xs + v;
                const bool colok = v >= R && v < kTWV - R && x >= R && x < a.W - R;
                const size_t o = (size_t)y * a.W + (colok ? x : R);
                sxc[c] = a.Sx[o];
                fvxc[c] = __int2float_rn(a.Vx[o]);
                tc[c] = a.Tx[o];
                // searched disparities dw + j: j in [jlo, jhi] (guide range,
                // match column x - dmin - d - R >= 0)
                int glo = 0, ghi = a.D - 1;
                if (a.guide && colok) {
                    const uint32_t g = __ldg(&a.guide[(size_t)(y / kGuideBlock) * a.guide_gw + x / kGuideBlock]);
                    glo = int(g & 0xFFFFu);
                    ghi = min(int(g >> 16), a.D - 1);
                }
                const int jlo = max(glo - dw, 0), jhi = min(min(ghi, x - a.dmin - R) - dw, kDPW - 1);
                const uint32_t smask = (colok && jlo <= jhi) ? ((2u << jhi) - (1u << jlo)) : 0u;
                float val[kDPW];
                float emax = -INFINITY;
#pragma unroll
                for (int j = 0; j < kDPW; ++j) {
                    const int kk = c - j + kDPW - 1;
                    const int num = n * C[j][c] - sxc[c] * syk[kk];
                    const float e = vyk[kk] >= tc[c] ? __fmul_rn(__int2float_rn(num), ryk[kk]) : 0.0f;
                    val[j] = (smask >> j) & 1u ? e : -INFINITY;
                    emax = fmaxf(emax, val[j]);
                }
                uint32_t cm = 0;
                const float thr = emax - fabsf(emax) * 2e-5f;
#pragma unroll
                for (int j = 0; j < kDPW; ++j) cm |= uint32_t(val[j] >= thr) << j;
                cm &= smask;
                const int j1 = __ffs(cm) - 1;
                if (emax == 0.0f) {  // every candidate scores +0: the lowest d wins
                    best[c] = ((unsigned long long)ordered(0.0f) << 32) | (0xFFFFFFFFu - uint32_t(dw + j1));
                    cand[c] = 0;
                } else {
                    best[c] = cm ? exact_key(c, j1) : 0ull;
                    cand[c] = cm & (cm - 1);
                }
            }
            // near-ties: every other disparity within the margin (rare)
            while (__any_sync(0xffffffffu, (cand[0] | cand[1] | cand[2] | cand[3]) != 0)) {
#pragma unroll
                for (int c = 0; c < kCPT; ++c)
                    if (cand[c]) {
                        const int j = __ffs(cand[c]) - 1;
                        cand[c] &= cand[c] - 1;
                        const unsigned long long key = exact_key(c, j);
                        best[c] = key > best[c] ? key : best[c];
                    }
            }
#pragma unroll
            for (int c = 0; c < kCPT; ++c)
                if (best[c]) atomicMax(&sKey[oy * TWO + 4 * lane + c - R], best[c]);
        }
    }
    __syncthreads();
    const bool direct = gridDim.z == 1;
    for (int idx = tid; idx < a.th * TWO; idx += kNT) {
        const int oy = idx / TWO, ox = idx - oy * TWO;
        const int x = xs + R + ox, y = y0 + oy;
        if (x >= a.W || y >= a.H) continue;
        const unsigned long long key = sKey[idx];
        if (direct) {
            const bool valid = x >= R && x < a.W - R && y >= R && y < a.H - R;
            store_ncc(a, x, y, valid, key);
        } else if (key) {
            atomicMax(&a.keys[(size_t)y * a.W + x], key);
        }
    }
    if (direct) return;
    // D split over gridDim.z CTAs: the last of the (strip, column tile) group
    // to finish writes the merged keys as the outputs and resets keys and
    // counter. Writers fence before counting; the merger fences after.
    __threadfence();
    __syncthreads();
    int* last = reinterpret_cast<int*>(bar + 1);
    if (tid == 0) {
        uint32_t* ctr = &a.counters[blockIdx.y * gridDim.x + blockIdx.x];
        const bool l = atomicAdd(ctr, 1u) == gridDim.z - 1;
        if (l) *ctr = 0u;
        *last = l;
    }
    __syncthreads();
    if (!*last) return;
    __threadfence();
    for (int idx = tid; idx < a.th * TWO; idx += kNT) {
        const int oy = idx / TWO, ox = idx - oy * TWO;
        const int x = xs + R + ox, y = y0 + oy;
        if (x >= a.W || y >= a.H) continue;
        unsigned long long* kp = &a.keys[(size_t)y * a.W + x];
        const unsigned long long key = __ldcg(kp);
        *kp = 0ull;
        const bool valid = x >= R && x < a.W - R && y >= R && y < a.H - R;
        store_ncc(a, x, y, valid, key);
    }
}

}  // namespace ncc
}  // namespace ct

#include "ncc_tc.cuh"

namespace ct {
namespace {

struct NccHandle : ct_handle {
    NccHandle() : ct_handle(Kind::BmNcc) {}
    ~NccHandle() override {
        if (device >= 0) cudaSetDevice(device);
        cudaFree(stats);
        cudaFree(keys);
        cudaFree(guide);
        cudaFree(counters);
    }
    ct_format fmt{};
    ct_ncc_params par{};
    int32_t* stats = nullptr;  // Sx, Vx, Sy, Vy, Tx
    unsigned long long* keys = nullptr;
    uint32_t* guide = nullptr;  // guided mode: one search range per 16 x 16 block
    uint32_t* counters = nullptr;  // one per (strip, column tile) at the smallest strip height
    int th = 32;
    int tensor_cores = 1;  // unguided matching: window cross sums on the tensor cores (ncc_tc_kernel)
    int th_tc = 64;        // its strip height
};

template <int R>
int launch_ncc(NccHandle* h, const ct_image* disp, const ct_image* score, const ct_image* L, const ct_image* Rr,
               const ct_image* init, cudaStream_t s) {
    using namespace ncc;
    static bool attr = false;
    if (!attr) {
        CT_CUDA_TRY(cudaFuncSetAttribute(ncc_match_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem_bytes(64, R)));
        attr = true;
    }
    const int W = h->fmt.width, H = h->fmt.height;
    const size_t N = (size_t)W * H;
    Args a{};
    a.W = W; a.H = H; a.D = h->par.disp_count; a.th = h->th;
    a.dmin = h->par.disp_min;
    a.Sx = h->stats; a.Vx = h->stats + N; a.Sy = h->stats + 2 * N; a.Vy = h->stats + 3 * N;
    a.Tx = h->stats + 4 * N;
    a.keys = h->keys;
    a.counters = h->counters;
    a.out = disp->ptr; a.out_pitch = disp->pitch_bytes; a.out_type = disp->type;
    a.score = score ? static_cast<float*>(score->ptr) : nullptr;
    a.score_pitch = score ? score->pitch_bytes : 0;
    a.status = h->d_status;
    if (init) {
        const int gw = (W + kGuideBlock - 1) / kGuideBlock, gh = (H + kGuideBlock - 1) / kGuideBlock;
        guide::range_kernel<<<dim3((gw + 127) / 128, gh), 128, 0, s>>>(init->ptr, init->pitch_bytes, init->type,
                                                                       W / init->width, W, H, h->guide, gw, gh,
                                                                       a.dmin);
        CT_LAUNCH_CHECK();
        a.guide = h->guide;
        a.guide_gw = gw;
    }
    dim3 sb(32, 8), sg((W + 31) / 32, (H + 63) / 64, 2);
    box_stats_kernel<R><<<sg, sb, 0, s>>>(static_cast<const uint8_t*>(L->ptr), L->pitch_bytes,
                                          static_cast<const uint8_t*>(Rr->ptr), Rr->pitch_bytes, W, H, h->stats,
                                          h->stats + N, h->stats + 4 * N, h->stats + 2 * N, h->stats + 3 * N);
    CT_LAUNCH_CHECK();
    if (!init && h->tensor_cores) {
        static bool attr_tc = false;
        if (!attr_tc) {
            CT_CUDA_TRY(cudaFuncSetAttribute(ncc_tc_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             tc::smem_bytes<R>()));
            attr_tc = true;
        }
        a.th = h->th_tc;
        dim3 grid((W + tc::kM - 1) / tc::kM, (H + a.th - 1) / a.th, (a.D + tc::kDB - 1) / tc::kDB);
        ncc_tc_kernel<R><<<grid, tc::kNT, tc::smem_bytes<R>(), s>>>(static_cast<const uint8_t*>(L->ptr), L->pitch_bytes,
                                                         static_cast<const uint8_t*>(Rr->ptr), Rr->pitch_bytes, a);
        CT_LAUNCH_CHECK();
        return gate_launch(disp, score, L, 0, 2 * R + 1, h->grad_thresh, s);  // EvalGrad (NCC.cu:388-413)
    }
    const int NR = a.th + 2 * R;
    CUtensorMap tb, tm;
    if (int rc = make_tmap_2d(&tb, L->ptr, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, W, H, L->pitch_bytes, kBW, NR)) return rc;
    if (int rc = make_tmap_2d(&tm, Rr->ptr, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, W, H, Rr->pitch_bytes, kMWs, NR))
        return rc;
    dim3 grid((W + two_of(R) - 1) / two_of(R), (H + a.th - 1) / a.th, (a.D + kDPC - 1) / kDPC);
    ncc_match_kernel<R><<<grid, kNT, smem_bytes(a.th, R), s>>>(tb, tm, a);
    CT_LAUNCH_CHECK();
    return gate_launch(disp, score, L, 0, 2 * R + 1, h->grad_thresh, s);  // EvalGrad (NCC.cu:388-413)
}

}  // namespace
}  // namespace ct

using namespace ct;

extern "C" {

int ct_bm_ncc_create(ct_handle** out) {
    clear_error();
    if (!out) return fail(CT_EINVAL, "null output handle pointer");
    *out = new NccHandle();
    return CT_OK;
}

int ct_bm_ncc_configure(ct_handle* hh, int32_t device, const ct_format* fmt, const ct_ncc_params* p) {
    clear_error();
    auto* h = (hh && hh->kind == Kind::BmNcc) ? static_cast<NccHandle*>(hh) : nullptr;
    if (!h) return fail(CT_ESTATE, "not an NCC matcher handle");
    if (!fmt || !p) return fail(CT_EINVAL, "null format or parameters");
    if (fmt->type != CT_PIX_U8) return fail(CT_ETYPE, "matcher input must be U8 (TPixel_Lum_UInt8)");
    if (fmt->width < 16 || fmt->height < 16 || fmt->width > 32768 || fmt->height > 32768)
        return fail(CT_EINVAL, "image size out of range (16..32768)");
    if (p->disp_count < 1 || p->disp_count > 256) return fail(CT_EINVAL, "disp_count must be 1..256");
    if (p->radius != 2 && p->radius != 4 && p->radius != 5)
        return fail(CT_EINVAL, "radius must be 5 (Patch_11x11), 4 (Patch_9x9) or 2 (Patch_5x5)");
    if (p->left_to_right != 1) return fail(CT_EINVAL, "the NCC matcher is left-to-right only");
    if (p->disp_min < 0 || p->disp_min + p->disp_count > 0xFFEF)
        return fail(CT_EINVAL, "disp_min must be >= 0 with disp_min + disp_count <= 65519");
    if (int rc = use_device(device)) return rc;
    cudaFree(h->stats); cudaFree(h->keys); cudaFree(h->guide); cudaFree(h->counters);
    h->stats = nullptr; h->keys = nullptr; h->guide = nullptr; h->counters = nullptr;
    h->device = device;
    if (int rc = h->init_status()) return rc;
    const size_t N = (size_t)fmt->width * fmt->height;
    if (cudaMalloc(&h->stats, 5 * N * sizeof(int32_t)) != cudaSuccess) return fail(CT_ENOMEM, "stats scratch");
    if (cudaMalloc(&h->keys, N * sizeof(unsigned long long)) != cudaSuccess) return fail(CT_ENOMEM, "key scratch");
    CT_CUDA_TRY(cudaMemset(h->keys, 0, N * sizeof(unsigned long long)));
    const size_t G = size_t((fmt->width + ncc::kGuideBlock - 1) / ncc::kGuideBlock) *
                     ((fmt->height + ncc::kGuideBlock - 1) / ncc::kGuideBlock);
    if (cudaMalloc(&h->guide, G * sizeof(uint32_t)) != cudaSuccess) return fail(CT_ENOMEM, "guide ranges");
    {  // merge counters for every strip height the configuration below may pick (>= 8 rows)
        const size_t C = size_t((fmt->width + ncc::two_of(p->radius) - 1) / ncc::two_of(p->radius)) *
                         ((fmt->height + 7) / 8);
        if (cudaMalloc(&h->counters, C * sizeof(uint32_t)) != cudaSuccess) return fail(CT_ENOMEM, "merge counters");
        CT_CUDA_TRY(cudaMemset(h->counters, 0, C * sizeof(uint32_t)));
    }
    h->fmt = *fmt;
    h->par = *p;
    {  // strip height: 32 rows (measured faster at 1080p than the taller strips
       // of fewer waves); lower only while the grid would not fill one wave of
       // 2 CTAs per SM
        const int two = ncc::two_of(p->radius), sms = sm_count(device);
        const long tiles = long((fmt->width + two - 1) / two) * ((p->disp_count + ncc::kDPC - 1) / ncc::kDPC);
        h->th = 32;
        while (h->th > 8 && tiles * ((fmt->height + h->th - 1) / h->th) < 2L * sms) h->th -= 2;
        // tensor-core kernel (one CTA per SM): the strip height minimising
        // waves x (rows + the strip's first window, worth ~6 rows)
        const long tiles_tc = long((fmt->width + ncc::tc::kM - 1) / ncc::tc::kM) *
                              ((p->disp_count + ncc::tc::kDB - 1) / ncc::tc::kDB);
        long best = -1;
        for (int th = 16; th <= 256; ++th) {
            const long ctas = tiles_tc * ((fmt->height + th - 1) / th);
            const long cost = ((ctas + sms - 1) / sms) * (th + 6);
            if (best < 0 || cost < best) { best = cost; h->th_tc = th; }
        }
    }
    h->configured = true;
    return CT_OK;
}

int ct_bm_ncc_set_tensor_cores(ct_handle* hh, int32_t enable) {
    clear_error();
    auto* h = (hh && hh->kind == Kind::BmNcc) ? static_cast<NccHandle*>(hh) : nullptr;
    if (!h) return fail(CT_ESTATE, "not an NCC matcher handle");
    if (enable != 0 && enable != 1) return fail(CT_EINVAL, "enable must be 0 or 1");
    h->tensor_cores = enable;
    return CT_OK;
}

int ct_bm_ncc_process(ct_handle* hh, const ct_image* disp, const ct_image* score, const ct_image* left,
                      const ct_image* right, const ct_image* disp_init, ct_stream stream) {
    clear_error();
    auto* h = (hh && hh->kind == Kind::BmNcc) ? static_cast<NccHandle*>(hh) : nullptr;
    if (!h) return fail(CT_ESTATE, "not an NCC matcher handle");
    if (!h->configured) return fail(CT_ESTATE, "process before configure");
    if (int rc = check_image(left, "left", 1u << CT_PIX_U8)) return rc;
    if (int rc = check_image(right, "right", 1u << CT_PIX_U8)) return rc;
    if (int rc = check_same_size(left, right, "left", "right")) return rc;
    if (left->width != h->fmt.width || left->height != h->fmt.height)
        return fail(CT_EFORMAT, "image size differs from the configured format");
    if (int rc = check_image(disp, "disp", (1u << CT_PIX_U8) | (1u << CT_PIX_U16))) return rc;
    if (int rc = check_same_size(disp, left, "disp", "left")) return rc;
    if (disp->type == CT_PIX_U8 && h->par.disp_min + h->par.disp_count > 255)
        return fail(CT_ETYPE, "U8 maps need disp_min + disp_count <= 255");
    if (score) {
        if (int rc = check_image(score, "score", 1u << CT_PIX_F32)) return rc;
        if (int rc = check_same_size(score, left, "score", "left")) return rc;
    }
    if (disp_init) {  // guided: coarse map at 1/s of the width, s a whole number
        if (int rc = check_image(disp_init, "disp_init", (1u << CT_PIX_U8) | (1u << CT_PIX_U16))) return rc;
        const int sc = disp_init->width > 0 ? left->width / disp_init->width : 0;
        if (sc < 1 || sc * disp_init->width != left->width)
            return fail(CT_EFORMAT, "disp_init width must divide the image width (scale %d / %d)", left->width,
                        disp_init->width);
        if (disp_init->height < (left->height + sc - 1) / sc)
            return fail(CT_EFORMAT, "disp_init needs at least ceil(height / %d) = %d rows", sc,
                        (left->height + sc - 1) / sc);
    }
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    switch (h->par.radius) {
        case 2: return launch_ncc<2>(h, disp, score, left, right, disp_init, s);
        case 4: return launch_ncc<4>(h, disp, score, left, right, disp_init, s);
        default: return launch_ncc<5>(h, disp, score, left, right, disp_init, s);
    }
}

}  // extern "C"
