// match_ad.cu — absolute-difference block matchers:
//   BlockMatcherSAD1::CDriver (exhaustive (2r+1)^2 SAD + WTA) and
//   BlockMatcherAW1/AW2 (best of 5 shifted 7x7 SAD windows + WTA + FP32
//   parabolic sub-pixel refinement).
//
// Layout (same decomposition as the census matcher): a CTA owns 128 "V
// columns" x th output rows x 64 disparities; warp w owns DPW = 4 or 8
// disparities (16 or 8 warps) and lane L the 4 adjacent columns 4L..4L+3. The uint8 image strips the CTA needs
// (th + 2*ext rows of the base view, 128 + 16 columns; of the match view,
// 192 + 16 columns) are staged in shared memory by two 2D TMA loads. Each
// thread walks the strip downwards keeping vertical running sums of |B - M|
// for 4 columns x 8 disparities packed as 16-bit pairs; the row leaving the
// window is recomputed from the staged pixels (cheaper than a register ring
// for a 1-byte cost). The horizontal pass takes r halo columns from the
// neighbouring lanes by shuffles (AlgoArraySum_W32H16::SumCache's two passes,
// Kernel.Algo.ArraySum_W32H16.h:163-200).
// The AW variant stores each row of 7x7 box sums S in a 7-row shared-memory
// ring and takes A = min(S(x,y), S(x-3,y), S(x+3,y), S(x,y-3), S(x,y+3)) with
// two packed 3-way mins (the min-variant of AlgoAdaptWnd3D's neighbourhood
// evaluation, Kernel.Algo.AdaptWnd3D.h:244-300, with the 5-window layout).
// Winner-take-all keys are (cost << 16 | d): the lowest cost wins, then the
// lowest d; warps merge through shared-memory atomicMin, CTAs that split D
// through a global key buffer.
#include "ct_internal.h"
#include "ct_device.cuh"
#include "guide.cuh"

namespace ct {
namespace ad {

constexpr int kCPT = 4, kTWV = 128, kDPC = 64;
constexpr int kPairs = kDPC / 2;         // disparity pairs per CTA (two disparities per 32-bit register)
// Disparities per warp DPW (4: 16 warps, 8: 8 warps per CTA; the kernel is
// instantiated for both): warps, threads, pairs per thread, match columns a
// thread reads per row.
__host__ __device__ constexpr int nt_of(int dpw) { return kDPC / dpw * 32; }
constexpr int kBW = kTWV + 16;        // staged base columns
constexpr int kMWs = kTWV + kDPC + 16; // staged match columns (208)
constexpr int kRing = 7;              // AW: rows of S kept
constexpr int kRingW = kTWV + 8;      // AW: padded ring row (4 words each side)

// Per-pixel costs are formed two disparities at a time in the 16-bit halves
// of a register as max(b + 256 - m, m + 256 - b) = |b - m| + 256 (no borrow
// crosses the halves); the 256 cancels in the running sums' add/subtract
// pairs, so every box sum carries (2r+1)^2 * 256 on top of the SAD (at most
// 81 * 511 = 41391 for 9x9: the 16-bit cost field never reaches 0xFFFF, the
// "no disparity" marker). The winner's cost in a key is biased by that much.
constexpr uint32_t kAbsBias = 0x01000100u;
__host__ __device__ constexpr int box_bias(int R) { return (2 * R + 1) * (2 * R + 1) * 256; }
static_assert(81 * 511 < 0xFFFF, "biased 9x9 box sums fit the 16-bit cost field");

__host__ __device__ constexpr int ext_of(int R, bool aw) { return aw ? 2 * R : R; }
__host__ __device__ constexpr int two_of(int R, bool aw) { return kTWV - 2 * ext_of(R, aw); }

struct Args {
    int W, H, D, th;
    int dmin;               // relative d matches column x -/+ (dmin + d); maps store dmin + d
    const uint32_t* guide;  // AW guided mode: search range per 16 x 16 block (guide.cuh), or null
    int guide_gw;
    uint32_t* keys;      // global keys when gridDim.z > 1 (or always for AW)
    void* out;
    size_t out_pitch;
    int out_type;
    int32_t* status;
};

__host__ __device__ constexpr size_t strip_bytes(int th, int R, bool aw) {
    return (size_t(kBW) * (th + 2 * ext_of(R, aw)) + 127) / 128 * 128 +
           (size_t(kMWs) * (th + 2 * ext_of(R, aw)) + 127) / 128 * 128;
}
__host__ __device__ constexpr size_t smem_bytes(int th, int R, bool aw) {
    return strip_bytes(th, R, aw) + (aw ? size_t(kRing) * kPairs * kRingW * 4 : 0) +
           size_t(th) * two_of(R, aw) * 4 + 16;
}

__device__ __forceinline__ int floor16(int v) { return v & ~15; }

// U8 / U16 / F32 disparity store from a (cost << 16 | d) key, d relative to
// dmin; 0xFFFF cost = none.
__device__ __forceinline__ void store_key(void* out, size_t pitch, int type, int x, int y, bool valid,
                                          uint32_t key, int dmin) {
    const bool ok = valid && (key >> 16) != 0xFFFFu;
    const uint32_t d = (key & 0xFFFFu) + uint32_t(dmin);
    char* row = static_cast<char*>(out) + (size_t)y * pitch;
    if (type == CT_PIX_U8) reinterpret_cast<uint8_t*>(row)[x] = ok ? uint8_t(d) : uint8_t(0xFF);
    else if (type == CT_PIX_U16) reinterpret_cast<uint16_t*>(row)[x] = ok ? uint16_t(d + 1) : uint16_t(0xFFFF);
    else reinterpret_cast<float*>(row)[x] = ok ? float(d) : -1.0f;
}

// Horizontal (2R+1)-wide sums of the packed column sums V of this lane's 4
// columns, halo columns taken from the neighbouring lanes.
template <int R>
__device__ __forceinline__ void hsum(const uint32_t (&V)[kCPT], uint32_t (&C)[kCPT]) {
    uint32_t win[kCPT + 2 * R];
#pragma unroll
    for (int j = 0; j < R; ++j) {  // column j - R < 0
        const int i = R - 1 - j;    // halo index: column -(i+1)
        win[j] = __shfl_up_sync(0xffffffffu, V[3 - (i % 4)], i / 4 + 1);
    }
#pragma unroll
    for (int c = 0; c < kCPT; ++c) win[R + c] = V[c];
#pragma unroll
    for (int i = 0; i < R; ++i) win[R + kCPT + i] = __shfl_down_sync(0xffffffffu, V[i % 4], i / 4 + 1);
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j <= 2 * R; ++j) s += win[j];
    C[0] = s;
#pragma unroll
    for (int c = 1; c < kCPT; ++c) {
        s = s + win[c + 2 * R] - win[c - 1];
        C[c] = s;
    }
}

template <int R, bool AW, int DIR, bool G, int DPW>  // G: guided (AW only)
__global__ void __launch_bounds__(nt_of(DPW), 1)
    ad_match_kernel(const __grid_constant__ CUtensorMap tmB, const __grid_constant__ CUtensorMap tmM, Args a) {
    constexpr int kDPW = DPW, kNW = kDPC / DPW, kNT = nt_of(DPW), kNP = DPW / 2, kMC = kCPT + DPW - 1;
    static_assert(kNW * kNP == kPairs, "pairs per CTA");
    constexpr int EXT = ext_of(R, AW);
    constexpr int TWO = two_of(R, AW);
    extern __shared__ __align__(128) unsigned char smem[];
    const int NR = a.th + 2 * EXT;
    uint8_t* sB = smem;
    uint8_t* sM = smem + (size_t(kBW) * NR + 127) / 128 * 128;
    unsigned char* after = smem + strip_bytes(a.th, R, AW);
    uint32_t* ring = reinterpret_cast<uint32_t*>(after);  // AW only
    uint32_t* sKey = reinterpret_cast<uint32_t*>(after + (AW ? size_t(kRing) * kNW * kNP * kRingW * 4 : 0));
    uint64_t* bar = reinterpret_cast<uint64_t*>(sKey + a.th * TWO);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int xs = blockIdx.x * TWO - EXT;
    const int y0 = blockIdx.y * a.th;
    for (int i = tid; i < a.th * TWO; i += kNT) sKey[i] = 0xFFFFFFFFu;
    // Guided (AW, left-to-right): disparity block z covers base + z kDPC ..,
    // base at the low end (rounded down to kDPW) of the union of the search
    // ranges of the 16 x 16 blocks this tile's outputs fall in; warps outside
    // the union skip the matching. Unguided, base = 0 and every warp below D
    // matches.
    int base = 0, ulo = 0, uhi = a.D - 1;
    if constexpr (G) {
        const int2 u = guide::tile_union(a.guide, a.guide_gw, xs + EXT, min(xs + EXT + TWO, a.W) - 1, y0,
                                         min(y0 + a.th, a.H) - 1, reinterpret_cast<int*>(bar + 1));
        ulo = u.x;
        uhi = min(u.y, a.D - 1);
        if (ulo <= uhi) base = ulo & ~(kDPW - 1);
    }
    const int dz0 = base + int(blockIdx.z) * kDPC;
    const int dw = dz0 + warp * kDPW;
    const bool warp_active = dw < a.D && ulo <= uhi && dw <= uhi && dw + kDPW - 1 >= ulo;
    const int ab = floor16(xs);
    const int am = DIR == 0 ? floor16(xs - a.dmin - dz0 - (kDPC - 1)) : floor16(xs + a.dmin + dz0);
    // AW windows reach EXT = 6 columns; SAD ones r columns.
    const bool interior = (dz0 + kDPC <= a.D) &&
                          (DIR == 0 ? (xs + EXT - EXT - a.dmin >= dz0 + kDPC - 1)
                                    : (xs + kTWV - 1 - EXT + a.dmin + dz0 + kDPC - 1 + EXT <= a.W - 1));

    if (tid == 0) {
        dev::prefetch_tmap(&tmB);
        dev::prefetch_tmap(&tmM);
        dev::mbar_init(bar, 1);
        dev::fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0) {
        dev::mbar_arrive_expect_tx(bar, uint32_t(kBW * NR + kMWs * NR));
        dev::tma_load_2d(sB, &tmB, ab, y0 - EXT, bar);
        dev::tma_load_2d(sM, &tmM, am, y0 - EXT, bar);
    }
    const bool got = dev::mbar_wait_bounded(bar, 0);
    if (__syncthreads_or(!got)) {
        if (tid == 0) dev::report(a.status, CT_ETIMEOUT);
        return;
    }

    const int bo = xs - ab + 4 * lane;                                        // base column 0 in strip
    const int mo = DIR == 0 ? (xs - a.dmin - dz0 - am) + 4 * lane - kDPW * warp - (kDPW - 1)  // (c=0, j=kDPW-1)
                            : (xs + a.dmin + dz0 - am) + 4 * lane + kDPW * warp;                // (c=0, j=0)
    uint32_t dlo[kNP];
#pragma unroll
    for (int p = 0; p < kNP; ++p) dlo[p] = uint32_t(dw + 2 * p);

    auto row_pairs = [&](int i, uint32_t (&P)[kCPT][kNP]) {
        const uint8_t* rb = sB + i * kBW + bo;
        const uint8_t* rm = sM + i * kMWs + mo;
        uint32_t b2[kCPT], m2[kMC - 1];
#pragma unroll
        for (int c = 0; c < kCPT; ++c) b2[c] = uint32_t(rb[c]) * 0x10001u;  // b in both halves
        // match pixel pairs: the low half is disparity 2p of the pair, the
        // high half 2p + 1 (left-to-right: columns k0, k0 - 1; right-to-left:
        // k0, k0 + 1)
        {
            uint32_t m[kMC];
#pragma unroll
            for (int k = 0; k < kMC; ++k) m[k] = rm[k];
#pragma unroll
            for (int k = 0; k < kMC - 1; ++k) m2[k] = DIR == 0 ? m[k + 1] + (m[k] << 16) : m[k] + (m[k + 1] << 16);
        }
#pragma unroll
        for (int c = 0; c < kCPT; ++c)
#pragma unroll
            for (int p = 0; p < kNP; ++p) {
                const uint32_t mp = m2[DIR == 0 ? c - 2 * p + kDPW - 2 : c + 2 * p];
                P[c][p] = __vmaxu2(b2[c] + kAbsBias - mp, mp + kAbsBias - b2[c]);  // |b - m| + 256 per half
            }
    };

    uint32_t V[kNP][kCPT];  // [pair][column]
#pragma unroll
    for (int p = 0; p < kNP; ++p)
#pragma unroll
        for (int c = 0; c < kCPT; ++c) V[p][c] = 0;

    if (warp_active) {
        for (int i = 0; i < NR; ++i) {
            uint32_t Pn[kCPT][kNP];
            row_pairs(i, Pn);
            if (i >= 2 * R + 1) {
                uint32_t Po[kCPT][kNP];
                row_pairs(i - 2 * R - 1, Po);
#pragma unroll
                for (int c = 0; c < kCPT; ++c)
#pragma unroll
                    for (int p = 0; p < kNP; ++p) V[p][c] = V[p][c] + Pn[c][p] - Po[c][p];
            } else {
#pragma unroll
                for (int c = 0; c < kCPT; ++c)
#pragma unroll
                    for (int p = 0; p < kNP; ++p) V[p][c] += Pn[c][p];
            }
            if (i < 2 * R) continue;
            // S (box sums) of strip row i - R, all 4 pairs
            uint32_t S[kNP][kCPT];
#pragma unroll
            for (int p = 0; p < kNP; ++p) hsum<R>(V[p], S[p]);
            int oy;
            uint32_t A[kNP][kCPT];
            if (!AW) {
                oy = i - 2 * R;
#pragma unroll
                for (int p = 0; p < kNP; ++p)
#pragma unroll
                    for (int c = 0; c < kCPT; ++c) A[p][c] = S[p][c];
            } else {
                // S row index since the first S row: s = i - 2R; ring slot s % 7
                const int s = i - 2 * R;
                uint32_t* slot = ring + size_t(s % kRing) * kNW * kNP * kRingW;
#pragma unroll
                for (int p = 0; p < kNP; ++p)
                    *reinterpret_cast<uint4*>(slot + (warp * kNP + p) * kRingW + 4 + 4 * lane) =
                        make_uint4(S[p][0], S[p][1], S[p][2], S[p][3]);
                __syncwarp();
                if (s < 2 * R) continue;  // need S rows s - 3 and s - 6
                oy = s - 2 * R;
                const uint32_t* mid = ring + size_t((s - R) % kRing) * kNW * kNP * kRingW;
                const uint32_t* top = ring + size_t((s - 2 * R) % kRing) * kNW * kNP * kRingW;
#pragma unroll
                for (int p = 0; p < kNP; ++p) {
                    const uint32_t* rm = mid + (warp * kNP + p) * kRingW + 4 * lane;  // padded index of col 4L-4
                    const uint4 q0 = *reinterpret_cast<const uint4*>(rm);
                    const uint4 q1 = *reinterpret_cast<const uint4*>(rm + 4);
                    const uint4 q2 = *reinterpret_cast<const uint4*>(rm + 8);
                    const uint32_t w12[12] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w,
                                              q2.x, q2.y, q2.z, q2.w};  // cols 4L-4 .. 4L+7
                    const uint4 t = *reinterpret_cast<const uint4*>(top + (warp * kNP + p) * kRingW + 4 + 4 * lane);
                    const uint32_t tw[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
                    for (int c = 0; c < kCPT; ++c) {
                        const uint32_t m3 = dev::min3_u16x2(w12[4 + c], w12[4 + c - R], w12[4 + c + R]);
                        A[p][c] = dev::min3_u16x2(m3, tw[c], S[p][c]);
                    }
                }
            }
            if (oy < 0 || oy >= a.th) continue;
#pragma unroll
            for (int c = 0; c < kCPT; ++c) {
                const int v = 4 * lane + c;
                if (v < EXT || v >= kTWV - EXT) continue;
                uint32_t best = 0xFFFFFFFFu;
                const int x = xs + v;
                int lim = DIR == 0 ? x - EXT - a.dmin : a.W - 1 - EXT - x - a.dmin;
                lim = min(lim, a.D - 1);
                int glo = 0;
                if constexpr (G) {  // this pixel's block range (pixels outside the image search nothing)
                    const int y = y0 + oy;
                    const uint32_t g = (y < a.H && x < a.W)
                                           ? __ldg(&a.guide[(size_t)(y / guide::kBlock) * a.guide_gw + x / guide::kBlock])
                                           : 0x0000FFFFu;
                    glo = int(g & 0xFFFFu);
                    lim = min(lim, int(g >> 16));
                }
#pragma unroll
                for (int p = 0; p < kNP; ++p) {
                    uint32_t klo = __byte_perm(A[p][c], dlo[p], 0x1054);        // cost_lo << 16 | d
                    uint32_t khi = (A[p][c] & 0xFFFF0000u) | (dlo[p] + 1);       // cost_hi << 16 | d+1
                    if (!interior || G) {
                        if (int(dlo[p]) > lim || int(dlo[p]) < glo) klo |= 0xFFFF0000u;
                        if (int(dlo[p]) + 1 > lim || int(dlo[p]) + 1 < glo) khi |= 0xFFFF0000u;
                    }
                    best = min(best, min(klo, khi));
                }
                atomicMin(&sKey[oy * TWO + v - EXT], best);
            }
        }
    } else if (AW) {
        // inactive warps still own ring slices nobody reads; nothing to do
    }
    __syncthreads();
    const bool direct = !AW && gridDim.z == 1;
    for (int idx = tid; idx < a.th * TWO; idx += kNT) {
        const int oy = idx / TWO, ox = idx - oy * TWO;
        const int x = xs + EXT + ox, y = y0 + oy;
        if (x >= a.W || y >= a.H) continue;
        const uint32_t key = sKey[idx];
        if (direct) {
            const bool valid = x >= EXT && x < a.W - EXT && y >= EXT && y < a.H - EXT;
            store_key(a.out, a.out_pitch, a.out_type, x, y, valid, key, a.dmin);
        } else {
            atomicMin(&a.keys[(size_t)y * a.W + x], key);
        }
    }
}

__global__ void ad_finalize_kernel(uint32_t* keys, int W, int H, int ext, void* out, size_t pitch, int type,
                                   int dmin) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    uint32_t* kp = &keys[(size_t)y * W + x];
    const uint32_t key = *kp;
    *kp = 0xFFFFFFFFu;
    const bool valid = x >= ext && x < W - ext && y >= ext && y < H - ext;
    store_key(out, pitch, type, x, y, valid, key, dmin);
}

// Sub-pixel refinement from the merged AW keys: with d the winner relative to
// dmin and e = dmin + d its disparity, e* = e + (c- - c+) / (2 (c- - 2 c0 + c+))
// in IEEE FP32, skipped at d = 0, d = D-1 or when e + 1 is not searchable
// (x - (e+1) - 6 < 0). c-, c+ are the AW costs at e - 1, e + 1: the minimum
// of the five 7x7 SADs centred at (x, y), (x -/+ 3, y), (x, y -/+ 3). Resets
// the keys.
// A CTA refines a 32 x 16 pixel tile (two rows per thread). It stages the
// base view's 28 rows x 64 columns around the tile and the match view's rows
// over the band of columns the tile's winners reach (at most 21 16-byte
// chunks for D <= 256), then
// each thread forms the 133 cells of its plus-shaped 13 x 13 neighbourhood
// with both disparities in the two 16-bit halves (|b - m| + 256, as in the
// matcher) and sums the five windows from partial column sums.
constexpr int kSpX = 32, kSpTY = 8, kSpQ = 2, kSpY = kSpTY * kSpQ;  // 32 x 16 pixels, 2 rows per thread
constexpr int kSpRows = kSpY + 12;
constexpr int kSpLCols = 64;                         // base columns x0 - 16 .. x0 + 47 (16-byte chunks)
constexpr int kSpRCols = 21 * 16;                    // match band rounded out to 16-byte chunks

__global__ void __launch_bounds__(kSpX * kSpTY) aw_subpixel_kernel(uint32_t* keys, int W, int H, int D, int dmin,
                                                                 const uint8_t* L, size_t pl, const uint8_t* Rm,
                                                                 size_t pr, void* out, size_t pitch, int type) {
    __shared__ __align__(16) uint8_t sL[kSpRows][kSpLCols];
    __shared__ __align__(16) uint8_t sR[kSpRows][kSpRCols];
    __shared__ int sRange[2];
    const int tx = threadIdx.x, tid = threadIdx.y * kSpX + tx;
    const int x0 = blockIdx.x * kSpX, y0 = blockIdx.y * kSpY;
    const int x = x0 + tx;
    if (tid == 0) {
        sRange[0] = 0x7FFFFFFF;
        sRange[1] = -0x7FFFFFFF;
    }
    // this thread's pixels: rows ty = threadIdx.y + 8 q of the tile
    uint32_t key[kSpQ];
    bool need[kSpQ];
    int lo = 0x7FFFFFFF, hi = -0x7FFFFFFF;
#pragma unroll
    for (int q = 0; q < kSpQ; ++q) {
        const int y = y0 + threadIdx.y + kSpTY * q;
        const bool inb = x < W && y < H;
        key[q] = 0xFFFFFFFFu;
        if (inb) {
            uint32_t* kp = &keys[(size_t)y * W + x];
            key[q] = *kp;
            *kp = 0xFFFFFFFFu;
        }
        const bool valid = inb && x >= 6 && x < W - 6 && y >= 6 && y < H - 6 && (key[q] >> 16) != 0xFFFFu;
        const int d = int(key[q] & 0xFFFFu);
        const int e = dmin + d;
        need[q] = type == CT_PIX_F32 && valid && d > 0 && d < D - 1 && x - (e + 1) - 6 >= 0;
        if (inb && !need[q]) {
            if (type != CT_PIX_F32 || !valid) store_key(out, pitch, type, x, y, valid, key[q], dmin);
            else reinterpret_cast<float*>(static_cast<char*>(out) + (size_t)y * pitch)[x] = float(e);
        }
        if (need[q]) {
            lo = min(lo, e);
            hi = max(hi, e);
        }
    }
    // Staging in 16-byte chunks (the images' rows start 16-byte aligned, as
    // their TMA maps require); a chunk reaching past the width is read byte
    // by byte, chunks outside the image read 0. The base tile (columns
    // x0 - 16 + c) does not depend on the winners: its loads go out with the
    // key loads, before the range reduction.
    auto chunk = [&](const uint8_t* img, size_t ip, int gy, int gx, uint8_t* dst) {
        uint4 v = make_uint4(0, 0, 0, 0);
        if (gy >= 0 && gy < H && gx >= 0 && gx < W) {
            const uint8_t* src = img + (size_t)gy * ip + gx;
            if (gx + 16 <= W) {
                v = *reinterpret_cast<const uint4*>(src);
            } else {
                uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
                for (int k = 0; k < 16; ++k)
                    if (gx + k < W) w[k >> 2] |= uint32_t(src[k]) << (8 * (k & 3));
                v = make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
        *reinterpret_cast<uint4*>(dst) = v;
    };
    for (int i = tid; i < kSpRows * (kSpLCols / 16); i += kSpX * kSpTY) {
        const int r = i / (kSpLCols / 16), j = i - r * (kSpLCols / 16);
        chunk(L, pl, y0 - 6 + r, x0 - 16 + 16 * j, &sL[r][16 * j]);
    }
    __syncthreads();  // sRange initialised
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    if ((tid & 31) == 0) {
        atomicMin(&sRange[0], lo);
        atomicMax(&sRange[1], hi);
    }
    __syncthreads();
    const int emin = sRange[0], emax = sRange[1];
    if (emin > emax) return;  // no pixel of the tile is refined
    // match band: columns rs + c covering x0 - emax - 7 .. x0 + 38 - emin
    // (emax - emin <= D - 3 <= 253: at most 21 chunks)
    const int rs = (x0 - emax - 7) & ~15;
    const int nch = (x0 + 38 - emin - rs) / 16 + 1;
    for (int i = tid; i < kSpRows * nch; i += kSpX * kSpTY) {
        const int r = i / nch, j = i - r * nch;
        chunk(Rm, pr, y0 - 6 + r, rs + 16 * j, &sR[r][16 * j]);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kSpQ; ++q) {
        if (!need[q]) continue;
        const int ty = threadIdx.y + kSpTY * q, y = y0 + ty;
        const int e = dmin + int(key[q] & 0xFFFFu);
        // cell (r, k): row y - 6 + r, column x - 6 + k; base pixel sL[ty + r][tx + 10 + k];
        // match pixel of disparity e -/+ 1 at band column base + k + 2 / base + k
        const int base = x - e - 7 - rs;
        auto cell = [&](int r, int k) {
            const uint32_t b2 = uint32_t(sL[ty + r][tx + 10 + k]) * 0x10001u;
            const uint32_t m2 = uint32_t(sR[ty + r][base + k + 2]) + (uint32_t(sR[ty + r][base + k]) << 16);
            return __vmaxu2(b2 + kAbsBias - m2, m2 + kAbsBias - b2);  // (|b - m-| + 256) | (|b - m+| + 256) << 16
        };
        // partial column sums: top rows 0-2, middle 3-5, centre 6, lower 7-9, bottom 10-12
        uint32_t mid[13], sl = 0, sc = 0, sr = 0, su = 0, sd = 0;
#pragma unroll
        for (int k = 0; k < 13; ++k) {
            uint32_t a = 0, m = cell(6, k), c = 0;
#pragma unroll
            for (int r = 3; r < 6; ++r) a += cell(r, k);
#pragma unroll
            for (int r = 7; r < 10; ++r) c += cell(r, k);
            mid[k] = a + m + c;
            if (k >= 3 && k <= 9) {
                uint32_t t = 0, b = 0;
#pragma unroll
                for (int r = 0; r < 3; ++r) t += cell(r, k);
#pragma unroll
                for (int r = 10; r < 13; ++r) b += cell(r, k);
                su += t + a + m;
                sd += m + c + b;
                sc += mid[k];
            }
        }
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            sl += mid[k];
            sr += mid[k + 6];
        }
        const uint32_t mn = __vminu2(__vminu2(__vminu2(sc, sl), __vminu2(sr, su)), sd);
        const int cm = int(mn & 0xFFFFu) - box_bias(3), cp = int(mn >> 16) - box_bias(3);
        const int c0 = int(key[q] >> 16) - box_bias(3);  // the winner's 7x7 AW cost (keys carry the box bias)
        float sp = float(e);
        const int den = cm - 2 * c0 + cp;
        if (den > 0) sp = __fadd_rn(float(e), __fdiv_rn(float(cm - cp), float(2 * den)));
        reinterpret_cast<float*>(static_cast<char*>(out) + (size_t)y * pitch)[x] = sp;
    }
}

}  // namespace ad

// ---------------------------------------------------------------------------
// Handles and C ABI
// ---------------------------------------------------------------------------
namespace {

struct AdHandle : ct_handle {
    explicit AdHandle(Kind k) : ct_handle(k) {}
    ~AdHandle() override {
        if (device >= 0) cudaSetDevice(device);
        cudaFree(keys);
        cudaFree(guide);
    }
    ct_format fmt{};
    int D = 0, R = 4, dir = 0, dmin = 0;
    uint32_t* keys = nullptr;
    uint32_t* guide = nullptr;  // AW guided mode: one search range per 16 x 16 block
    int th = 32;
};

template <int R, bool AW, int DIR, bool G, int DPW>
int set_attr() {
    static bool done = false;
    if (!done) {
        CT_CUDA_TRY(cudaFuncSetAttribute(ad::ad_match_kernel<R, AW, DIR, G, DPW>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)ad::smem_bytes(64, R, AW)));
        done = true;
    }
    return CT_OK;
}

// Disparities per warp: 4 (16 warps per CTA) for the adaptive windows and
// the SAD windows from 7x7 up, which are bound by instruction latency at one
// CTA per SM; 8 for the smaller SAD windows, where loading each base pixel
// for 8 disparities saves more than the extra warps hide (measured: AW
// 2560x1440 1.162 -> 1.025 ms and SAD 9x9 640x480 0.0266 -> 0.0245 ms with 4;
// SAD 5x5 1920x1080 0.1833 ms with 8 against 0.1933 with 4).
template <int R, bool AW>
constexpr int dpw_for() { return (AW || R >= 3) ? 4 : 8; }

template <int R, bool AW, int DIR>
int launch_ad(AdHandle* h, const ct_image* disp, const ct_image* L, const ct_image* Rimg, cudaStream_t s,
              const ct_image* init = nullptr) {
    using namespace ad;
    const bool guided = AW && init;  // the guided variant exists for the AW matcher only
    constexpr int DPW = dpw_for<R, AW>();
    if constexpr (AW) {
        if (int rc = guided ? set_attr<R, AW, DIR, true, DPW>() : set_attr<R, AW, DIR, false, DPW>()) return rc;
    } else {
        if (int rc = set_attr<R, AW, DIR, false, DPW>()) return rc;
    }
    const int W = h->fmt.width, H = h->fmt.height;
    constexpr int EXT = ext_of(R, AW), TWO = two_of(R, AW);
    Args a{};
    a.W = W; a.H = H; a.D = h->D; a.th = h->th;
    a.dmin = h->dmin;
    a.keys = h->keys;
    a.out = disp->ptr; a.out_pitch = disp->pitch_bytes; a.out_type = disp->type;
    a.status = h->d_status;
    if (guided) {
        const int gw = (W + guide::kBlock - 1) / guide::kBlock, gh = (H + guide::kBlock - 1) / guide::kBlock;
        guide::range_kernel<<<dim3((gw + 127) / 128, gh), 128, 0, s>>>(init->ptr, init->pitch_bytes, init->type,
                                                                       W / init->width, W, H, h->guide, gw, gh,
                                                                       h->dmin);
        CT_LAUNCH_CHECK();
        a.guide = h->guide;
        a.guide_gw = gw;
    }
    const int NR = a.th + 2 * EXT;
    const ct_image* B = DIR == 0 ? L : Rimg;
    const ct_image* M = DIR == 0 ? Rimg : L;
    CUtensorMap tb, tm;
    if (int rc = make_tmap_2d(&tb, B->ptr, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, W, H, B->pitch_bytes, kBW, NR)) return rc;
    if (int rc = make_tmap_2d(&tm, M->ptr, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, W, H, M->pitch_bytes, kMWs, NR)) return rc;
    dim3 grid((W + TWO - 1) / TWO, (H + a.th - 1) / a.th, (h->D + kDPC - 1) / kDPC);
    constexpr int NT = nt_of(DPW);
    if constexpr (AW) {
        if (guided)
            ad_match_kernel<R, AW, DIR, true, DPW><<<grid, NT, smem_bytes(a.th, R, AW), s>>>(tb, tm, a);
        else
            ad_match_kernel<R, AW, DIR, false, DPW><<<grid, NT, smem_bytes(a.th, R, AW), s>>>(tb, tm, a);
    } else {
        ad_match_kernel<R, AW, DIR, false, DPW><<<grid, NT, smem_bytes(a.th, R, AW), s>>>(tb, tm, a);
    }
    CT_LAUNCH_CHECK();
    const ct_image* base = DIR == 0 ? L : Rimg;
    if (AW) {
        aw_subpixel_kernel<<<dim3((W + kSpX - 1) / kSpX, (H + kSpY - 1) / kSpY), dim3(kSpX, kSpTY), 0, s>>>(
            h->keys, W, H, h->D, h->dmin, static_cast<const uint8_t*>(L->ptr), L->pitch_bytes,
            static_cast<const uint8_t*>(Rimg->ptr), Rimg->pitch_bytes, disp->ptr, disp->pitch_bytes, disp->type);
        CT_LAUNCH_CHECK();
    } else if (grid.z > 1) {
        ad_finalize_kernel<<<dim3((W + 255) / 256, H), 256, 0, s>>>(h->keys, W, H, EXT, disp->ptr,
                                                                    disp->pitch_bytes, disp->type, h->dmin);
        CT_LAUNCH_CHECK();
    }
    // EvalGrad: SAD1's mean gradient over its window, AW1's standard
    // deviation over the whole 13 x 13 extent of the five windows
    return gate_launch(disp, nullptr, base, AW ? 1 : 0, AW ? 2 * EXT + 1 : 2 * R + 1, h->grad_thresh, s);
}

// Strip height: each SM works through ceil(CTAs / SMs) strips of th + 2 ext
// staged rows; pick the th in 8 .. 64 that minimises that (small images get
// enough strips to reach every SM, large ones fewer redundant halo rows).
int pick_ad_strip_height(int W, int H, int D, int ext, int two, int sms) {
    const long tiles = long((W + two - 1) / two) * ((D + ad::kDPC - 1) / ad::kDPC);
    int best = 32;
    long best_cost = -1;
    for (int th = 8; th <= 64; th += 2) {
        const long ctas = tiles * ((H + th - 1) / th);
        const long cost = (ctas + sms - 1) / sms * long(min(th, H) + 2 * ext);
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = th;
        }
    }
    return best;
}

int configure_ad(AdHandle* h, int32_t device, const ct_format* fmt, int D, int R, int dir, int dmin) {
    if (fmt->type != CT_PIX_U8) return fail(CT_ETYPE, "matcher input must be U8 (TPixel_Lum_UInt8)");
    if (fmt->width < 16 || fmt->height < 16 || fmt->width > 32768 || fmt->height > 32768)
        return fail(CT_EINVAL, "image size %dx%d out of range (16..32768)", fmt->width, fmt->height);
    if (D < 1 || D > 256) return fail(CT_EINVAL, "disp_count must be 1..256");
    if (dmin < 0 || dmin + D > 0xFFEF) return fail(CT_EINVAL, "disp_min must be >= 0 with disp_min + disp_count <= 65519");
    if (int rc = use_device(device)) return rc;
    cudaFree(h->keys);
    cudaFree(h->guide);
    h->keys = nullptr;
    h->guide = nullptr;
    h->device = device;
    if (int rc = h->init_status()) return rc;
    if (cudaMalloc(&h->keys, (size_t)fmt->width * fmt->height * 4) != cudaSuccess)
        return fail(CT_ENOMEM, "key scratch");
    CT_CUDA_TRY(cudaMemset(h->keys, 0xFF, (size_t)fmt->width * fmt->height * 4));
    const size_t G = size_t((fmt->width + guide::kBlock - 1) / guide::kBlock) *
                     ((fmt->height + guide::kBlock - 1) / guide::kBlock);
    if (cudaMalloc(&h->guide, G * 4) != cudaSuccess) return fail(CT_ENOMEM, "guide ranges");
    h->fmt = *fmt;
    h->D = D;
    h->R = R;
    h->dir = dir;
    h->dmin = dmin;
    const bool aw = h->kind == Kind::BmAw;
    h->th = pick_ad_strip_height(fmt->width, fmt->height, D, ad::ext_of(R, aw), ad::two_of(R, aw), sm_count(device));
    h->configured = true;
    return CT_OK;
}

int check_io(AdHandle* h, const ct_image* disp, const ct_image* L, const ct_image* R, uint32_t disp_types) {
    if (!h->configured) return fail(CT_ESTATE, "process before configure");
    if (int rc = check_image(L, "left", 1u << CT_PIX_U8)) return rc;
    if (int rc = check_image(R, "right", 1u << CT_PIX_U8)) return rc;
    if (int rc = check_same_size(L, R, "left", "right")) return rc;
    if (L->width != h->fmt.width || L->height != h->fmt.height)
        return fail(CT_EFORMAT, "image size differs from the configured format");
    if (int rc = check_image(disp, "disp", disp_types)) return rc;
    if (int rc = check_same_size(disp, L, "disp", "left")) return rc;
    if (disp->type == CT_PIX_U8 && h->dmin + h->D > 255)
        return fail(CT_ETYPE, "U8 maps need disp_min + disp_count <= 255");
    return CT_OK;
}

}  // namespace
}  // namespace ct

using namespace ct;

extern "C" {

int ct_bm_sad_create(ct_handle** out) {
    clear_error();
    if (!out) return fail(CT_EINVAL, "null output handle pointer");
    *out = new AdHandle(Kind::BmSad);
    return CT_OK;
}

int ct_bm_sad_configure(ct_handle* hh, int32_t device, const ct_format* fmt, const ct_sad_params* p) {
    clear_error();
    auto* h = (hh && hh->kind == Kind::BmSad) ? static_cast<AdHandle*>(hh) : nullptr;
    if (!h) return fail(CT_ESTATE, "not a SAD matcher handle");
    if (!fmt || !p) return fail(CT_EINVAL, "null format or parameters");
    if (p->radius < 1 || p->radius > 4) return fail(CT_EINVAL, "radius must be 1..4 (3x3 .. 9x9)");
    return configure_ad(h, device, fmt, p->disp_count, p->radius, p->left_to_right ? 0 : 1, p->disp_min);
}

int ct_bm_sad_process(ct_handle* hh, const ct_image* disp, const ct_image* left, const ct_image* right,
                      ct_stream stream) {
    clear_error();
    auto* h = (hh && hh->kind == Kind::BmSad) ? static_cast<AdHandle*>(hh) : nullptr;
    if (!h) return fail(CT_ESTATE, "not a SAD matcher handle");
    if (int rc = check_io(h, disp, left, right, (1u << CT_PIX_U8) | (1u << CT_PIX_U16))) return rc;
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    const int k = h->R * 2 + h->dir;
    switch (k) {
        case 2: return launch_ad<1, false, 0>(h, disp, left, right, s);
        case 3: return launch_ad<1, false, 1>(h, disp, left, right, s);
        case 4: return launch_ad<2, false, 0>(h, disp, left, right, s);
        case 5: return launch_ad<2, false, 1>(h, disp, left, right, s);
        case 6: return launch_ad<3, false, 0>(h, disp, left, right, s);
        case 7: return launch_ad<3, false, 1>(h, disp, left, right, s);
        case 8: return launch_ad<4, false, 0>(h, disp, left, right, s);
        case 9: return launch_ad<4, false, 1>(h, disp, left, right, s);
        default: return fail(CT_EINVAL, "unsupported radius");
    }
}

int ct_bm_aw_create(ct_handle** out) {
    clear_error();
    if (!out) return fail(CT_EINVAL, "null output handle pointer");
    *out = new AdHandle(Kind::BmAw);
    return CT_OK;
}

int ct_bm_aw_configure(ct_handle* hh, int32_t device, const ct_format* fmt, const ct_aw_params* p) {
    clear_error();
    auto* h = (hh && hh->kind == Kind::BmAw) ? static_cast<AdHandle*>(hh) : nullptr;
    if (!h) return fail(CT_ESTATE, "not an AW matcher handle");
    if (!fmt || !p) return fail(CT_EINVAL, "null format or parameters");
    if (p->left_to_right != 1) return fail(CT_EINVAL, "the AW matcher is left-to-right only");
    if (p->reserved1) return fail(CT_EINVAL, "reserved field must be 0");
    return configure_ad(h, device, fmt, p->disp_count, 3, 0, p->disp_min);
}

int ct_bm_aw_process(ct_handle* hh, const ct_image* disp, const ct_image* left, const ct_image* right,
                     ct_stream stream) {
    clear_error();
    auto* h = (hh && hh->kind == Kind::BmAw) ? static_cast<AdHandle*>(hh) : nullptr;
    if (!h) return fail(CT_ESTATE, "not an AW matcher handle");
    if (int rc = check_io(h, disp, left, right, (1u << CT_PIX_U8) | (1u << CT_PIX_U16) | (1u << CT_PIX_F32)))
        return rc;
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    return launch_ad<3, true, 0>(h, disp, left, right, s);
}

int ct_bm_aw_process_guided(ct_handle* hh, const ct_image* disp, const ct_image* left, const ct_image* right,
                            const ct_image* disp_init, ct_stream stream) {
    clear_error();
    auto* h = (hh && hh->kind == Kind::BmAw) ? static_cast<AdHandle*>(hh) : nullptr;
    if (!h) return fail(CT_ESTATE, "not an AW matcher handle");
    if (int rc = check_io(h, disp, left, right, (1u << CT_PIX_U8) | (1u << CT_PIX_U16) | (1u << CT_PIX_F32)))
        return rc;
    if (int rc = check_image(disp_init, "disp_init", (1u << CT_PIX_U8) | (1u << CT_PIX_U16))) return rc;
    const int sc = left->width / disp_init->width;
    if (sc < 1 || sc * disp_init->width != left->width)
        return fail(CT_EFORMAT, "disp_init width must divide the image width (%d / %d)", left->width,
                    disp_init->width);
    if (disp_init->height < (left->height + sc - 1) / sc)
        return fail(CT_EFORMAT, "disp_init needs at least ceil(height / %d) = %d rows", sc,
                    (left->height + sc - 1) / sc);
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    return launch_ad<3, true, 0>(h, disp, left, right, s, disp_init);
}

}  // extern "C"
