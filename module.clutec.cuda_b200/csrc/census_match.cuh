// census_match.cuh — the fused census matcher kernel: Hamming cost (popcount
// of XOR of 64-bit descriptors) + 5x5 box aggregation + winner-take-all, one
// launch per direction.
//
// Mapping to B200:
//  * A CTA owns a tile of 128 "V columns" (124 output columns plus 2 halo
//    columns on each side) x th output rows x 64 disparities. Its warps share
//    the same columns and rows; warp w owns disparities dz0 + DPW w .. + DPW-1
//    (DPW = 4: 16 warps of <= 128 registers; DPW = 8: 8 warps) and lane L owns
//    the 4 adjacent columns 4L..4L+3.
//  * Descriptor rows are staged in shared memory by 2D TMA tile loads (one box
//    of 10 rows of the base view and one of the match view per batch), two
//    batches in flight, completion tracked by mbarriers with bounded waits;
//    one CTA barrier per batch.
//  * Each thread keeps, in registers, the vertical running sums V of its 4
//    columns x DPW disparities and a 5-deep ring of the per-row Hamming costs
//    (the role of AlgoArraySum_W32H16::SumCache's vertical pass,
//    Kernel.Algo.ArraySum_W32H16.h:163-182). Costs for two disparities are
//    packed in the two 16-bit halves of one register, so every add/sub of the
//    running sums handles two disparities.
//  * The horizontal pass (ArraySum_W32H16.h:186-200) takes the 2 halo columns
//    from the neighbouring lanes with warp shuffles and runs a 5-wide running
//    sum over the thread's columns.
//  * Rows are software-pipelined: the aggregation and winner-take-all of the
//    window ending at row i-1 are issued next to the popcounts of row i, so
//    the POPC pipe (16 lanes / clock / SM, the bound) is kept busy while the
//    integer pipes do the rest.
//  * Winner-take-all folds the disparity into the low 5 bits of each 16-bit
//    lane (key = C << 5 | d mod 32, C <= 25 * 63 = 1575 so it fits): the min
//    over a thread's disparities is one or two packed mins plus a half swap,
//    and the lowest d wins ties by construction (the reference's strict '<'
//    scanning d upward). Warps of one 32-disparity group merge with a
//    shared-memory atomicMin; the two groups of a CTA are merged, converted to
//    (C << 16 | d) and flushed after every batch, directly into the disparity
//    map when the CTA saw all D, else through a global atomicMin whose keys a
//    finalize kernel turns into disparities.
#pragma once

#include <cstdint>

#include "ct_device.cuh"

namespace ct {
namespace cm {

constexpr int kCPT = 4;                 // columns per thread
constexpr int kTWV = 32 * kCPT;         // 128 V columns per tile
constexpr int kAR = 2;                  // aggregation radius (5x5)
constexpr int kTWO = kTWV - 2 * kAR;    // 124 output columns per tile
constexpr int kDPC = 64;                // disparities per CTA
constexpr int kGroups = kDPC / 32;      // key groups of 32 disparities
constexpr int kRB = 2 * kAR + 1;        // ring depth = vertical window = 5
constexpr int kBR = 2 * kRB;            // cost rows per TMA batch = 10
constexpr int kMW = kTWV + kDPC;        // 192 match columns staged per row

// Descriptor scratch layout ("pair-planar"): each row holds the 16-byte pairs
// of adjacent columns (x & ~1, x | 1), even pairs in plane 0, odd pairs in
// plane 1: word (x, y) lives at y * pitch + ((x >> 1) & 1) * 2 * NI +
// (x >> 2) * 2 + (x & 1), NI = ceil(W / 4), pitch = 4 * NI. A lane's 4
// adjacent columns are then two 16-byte elements at consecutive indices of
// the two planes, so a warp's 16-byte shared loads are contiguous (no bank
// conflicts). Staged boxes: [row][plane][kPB or kPM][2] words.
constexpr int kPB = kTWV / 4 + 1;       // 33 pair indices per plane (base rows)
constexpr int kPM = kMW / 4 + 1;        // 49 (match rows)
constexpr int kRowB = 2 * kPB * 2;      // words per staged base row
constexpr int kRowM = 2 * kPM * 2;      // words per staged match row
constexpr int kStageB = (kBR * kRowB * 8 + 127) / 128 * 128;  // bytes per stage (128-aligned)
constexpr int kStageM = (kBR * kRowM * 8 + 127) / 128 * 128;
constexpr uint32_t kTxB = kBR * kRowB * 8;  // bytes a base box delivers
constexpr uint32_t kTxM = kBR * kRowM * 8;

__host__ __device__ constexpr int planar_ni(int W) { return (W + 3) / 4; }
__host__ __device__ constexpr size_t planar_pitch(int W) { return size_t(4) * planar_ni(W); }
__host__ __device__ constexpr size_t planar_index(int x, int y, int W) {
    return size_t(y) * planar_pitch(W) + size_t((x >> 1) & 1) * 2 * planar_ni(W) + size_t(x >> 2) * 2 + (x & 1);
}

// Variant: disparities per warp (8 = 8 warps of 255 registers, one CTA of 8
// warps per SM; 4 = 16 warps of at most 128 registers, 16 warps per SM).
template <int DPW>
struct Var {
    static constexpr int kNP = DPW / 2;           // packed pairs per thread
    static constexpr int kNW = kDPC / DPW;        // warps per CTA
    static constexpr int kNT = kNW * 32;          // threads per CTA
    static constexpr int kWords = DPW + 4;        // match descriptors a thread reads per row
    static constexpr int kWarpsPerGroup = 32 / DPW;
};

// When D spans several CTAs (gridDim.z > 1) their winners are merged either
// (merge_last = 1) through per-z key planes keys[z][y][x] written with plain
// stores, merged by whichever CTA of the (strip, column tile) group finishes
// last (one atomic counter per group, reset by that CTA), or (merge_last = 0)
// by atomicMin into one key plane that keys_finalize_kernel converts.
struct MatchArgs {
    int W, H, D;
    // Minimum disparity: relative disparity d is matched against column
    // x -/+ (dmin + d) and stored as dmin + d. dmin is even (the match rows
    // are read as column pairs); an odd minimum m runs as dmin = m - 1 with
    // dfirst = 1, which excludes relative d = 0, and D one larger.
    int dmin, dfirst;
    int th;             // output rows per CTA (strip height)
    uint32_t* keys;     // key plane(s), see above
    uint32_t* counters; // merge_last: one counter per (strip, column tile), 0 between calls
    int merge_last;
    void* out;          // disparity output
    size_t out_pitch;
    int out_type;       // CT_PIX_U8 / CT_PIX_U16
    int32_t* status;
    // Optional cost-curve volume (kernels instantiated with CURVE = true):
    // row (y, g) at curve + (y * curve_groups + g) * curve_pitch holds one
    // 32-bit word per pixel, word x + 2 for column x, whose bytes are the
    // codes of disparities 4g .. 4g + 3 (byte k = disparity 4g + k).
    // Code = aggregated cost >> 3 (at most 1575 >> 3 = 196); 255 for a
    // disparity whose match window leaves the image. Border pixels (within 2
    // of the image edge, which have no disparity) get unspecified codes.
    uint32_t* curve;
    size_t curve_pitch;  // 32-bit words per row, a multiple of 4
    int curve_groups;    // ceil(D / 4)
    // Fused right-to-left winner (left-to-right kernels instantiated with
    // RL = true): one key per right-view pixel, row y at rl_keys + y *
    // rl_pitch. The 5x5 Hamming cost of right pixel x_R at disparity e equals
    // the left-to-right cost of left pixel x_R + e at e (the same two
    // windows), so every cost this pass computes also bids for the right
    // view: key rl_tag | (C << 16) | e, e = dmin + d absolute, C < 2047.
    // rl_tag (bits 27..31) is one less on every call, so this call's bids are
    // below every key an earlier call left and the plane needs no reset pass
    // (rl_check_kernel ignores keys of another tag; the plane is set to
    // 0xFFFFFFFF again when the tag wraps).
    uint32_t* rl_keys;
    size_t rl_pitch;     // words, a multiple of 4
    uint32_t rl_tag;     // tag << 27
};

// Right-view key plane pitch for width W (words): rows 16-byte aligned.
__host__ __device__ constexpr size_t rl_pitch_words(int W) { return (size_t(W) + 3) / 4 * 4; }
constexpr int kRLTagShift = 27;
constexpr int kRLTags = 32;  // tags 31 .. 0, then the plane is reset

// Curve word pitch for width W: words 0 .. W + 1 used, rounded up to 64
// words (256 bytes) so every row starts 16-byte aligned.
__host__ __device__ constexpr size_t curve_pitch_words(int W) { return (size_t(W) + 2 + 63) / 64 * 64; }

// Shared memory: 2 stages of base (10 rows x 66 pairs) and match (10 x 98
// pairs) descriptors, 2 buffers x 2 groups x 10 rows x 128 key slots, 2
// mbarriers and a flag. 71.3 KB.
__host__ __device__ constexpr size_t smem_bytes() {
    return size_t(2) * (kStageB + kStageM) + size_t(2) * kGroups * kBR * kTWV * 4 + 2 * 8 + 16;
}
// The fused right-to-left keys: 2 buffers x kGroups x kBR rows x kRLW
// right-view columns (V columns minus the 64 disparities of the CTA), after
// the rest; one row set per group of 32 disparities, whose 16-bit keys carry
// d & 31 (as the left-to-right key buffers).
// Right-view index i of a row lives at word (i & 3) * kRLQ + (i >> 2): a
// thread's bids for one anti-diagonal are at i = 4 * lane + const, so the 32
// lanes' shared atomics hit 32 consecutive words (with i itself as the word
// index they would be 4-way bank conflicts).
constexpr int kRLW = kTWV + kDPC;  // 192 (191 used)
constexpr int kRLQ = kRLW / 4;
static_assert(kRLW % 4 == 0 && (kDPC - 1) % 4 == 3, "right-view key interleave");
__host__ __device__ constexpr int rl_word(int i) { return (i & 3) * kRLQ + (i >> 2); }
__host__ __device__ constexpr size_t rl_offset() { return (smem_bytes() + 127) / 128 * 128; }
__host__ __device__ constexpr size_t smem_bytes_rl() { return rl_offset() + size_t(2) * kGroups * kBR * kRLW * 4; }

// Disparity code for an output pixel from its merged key (C << 16 | d), d
// relative to dmin.
__device__ __forceinline__ void store_disp(void* out, size_t pitch, int type, int x, int y, bool valid,
                                           uint32_t key, int dmin = 0) {
    const uint32_t d = (key & 0xFFFFu) + uint32_t(dmin);
    const bool ok = valid && (key >> 16) < 2047u;
    if (type == 1) {  // CT_PIX_U8
        reinterpret_cast<uint8_t*>(static_cast<char*>(out) + (size_t)y * pitch)[x] = ok ? uint8_t(d) : uint8_t(0xFF);
    } else {  // CT_PIX_U16 (EDisparityId)
        reinterpret_cast<uint16_t*>(static_cast<char*>(out) + (size_t)y * pitch)[x] =
            ok ? uint16_t(d + 1) : uint16_t(0xFFFF);
    }
}

// A CTA's piece of work: column tile bx of nbx, strip by, disparity block bz
// of nbz. The single-image kernel takes it from blockIdx / gridDim; the
// batched persistent kernel from its work queue.
struct Tile {
    int bx, by, bz, nbx, nbz;
};

// Result of one tile: whether this CTA wrote final disparities for its
// (strip, column tile) group (always when nbz == 1; the last arriver
// otherwise), and whether a tile load timed out.
struct TileResult {
    bool group_done;
    bool aborted;
};

template <int DIR, bool EDGE, int DPW, bool CURVE, bool RL = false>
__device__ __forceinline__ TileResult match_body(const CUtensorMap* tmB, const CUtensorMap* tmM,
                                                 const MatchArgs& a, const Tile& t, uint64_t* sB, uint64_t* sM,
                                                 uint32_t* sKey, uint64_t* bars, int* sflag, const uint32_t* par,
                                                 int nb, int rows_here, int xs, int y0, int ye0, int dz0, int ms,
                                                 uint32_t* sKeyRL = nullptr) {
    static_assert(!RL || (DIR == 0 && !CURVE), "the fused right-to-left keys ride on the plain left-to-right pass");
    static_assert(!RL || DPW % 4 == 0, "the right-view key interleave assumes warps of 4k disparities");
    using VT = Var<DPW>;
    constexpr int NP = VT::kNP, NT = VT::kNT, NWD = VT::kWords;
    constexpr uint32_t kBytes = kTxB + kTxM;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int dw = dz0 + warp * DPW;
    const bool warp_active = dw < a.D;
    const int grp = warp / VT::kWarpsPerGroup;

    uint32_t V[kCPT][NP];
    uint32_t ring[kRB][kCPT][NP];
#pragma unroll
    for (int c = 0; c < kCPT; ++c)
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            V[c][p] = 0;
#pragma unroll
            for (int r = 0; r < kRB; ++r) ring[r][c][p] = 0;
        }
    uint32_t dconst[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p)
        dconst[p] = uint32_t((dw + 2 * p) & 31) | (uint32_t((dw + 2 * p + 1) & 31) << 16);
    int lim[kCPT];  // largest searchable d per column (EDGE tiles only)
#pragma unroll
    for (int c = 0; c < kCPT; ++c) {
        const int x = xs + 4 * lane + c;
        lim[c] = min(DIR == 0 ? x - kAR - a.dmin : a.W - 1 - kAR - x - a.dmin, a.D - 1);
    }
    // fused right-to-left: columns whose costs may not bid (the halo columns,
    // and columns whose window leaves the image on the right: right pixel
    // x - e must keep x - e + e + 2 <= W - 1) get key 0xFFFF in both halves
    uint32_t rlbad[kCPT];
#pragma unroll
    for (int c = 0; c < kCPT; ++c) {
        const int v = 4 * lane + c, x = xs + v;
        rlbad[c] = (v < kAR || v >= kAR + kTWO || x > a.W - 1 - kAR) ? 0xFFFFFFFFu : 0u;
    }
    // First match column this thread reads per row, as an (even) offset from
    // ms: its words are the pairs (ms + mstart) / 2 + u, u < NWD / 2.
    const int mstart = DIR == 0 ? 4 * lane + kDPC - DPW - DPW * warp : 4 * lane + DPW * warp;
    // Word offsets, within a staged row, of this thread's two base pairs and
    // its NWD / 2 match pairs (pair-planar layout; see kPB).
    const int P0 = xs >> 1, i0 = P0 >> 1;          // first base pair, first staged pair index
    const int Q0 = ms >> 1, j0 = Q0 >> 1;          // same for the match rows
    int boff[2], moff[NWD / 2];
#pragma unroll
    for (int t = 0; t < 2; ++t) boff[t] = (((P0 + t) & 1) * kPB + ((P0 + t) >> 1) - i0 + lane) * 2;
    {
        const int g0 = Q0 + ((mstart - 4 * lane) >> 1);  // pair of u = 0, minus 2 * lane
#pragma unroll
        for (int u = 0; u < NWD / 2; ++u) moff[u] = (((g0 + u) & 1) * kPM + ((g0 + u) >> 1) - j0 + lane) * 2;
    }

    // Adds cost row r of stage s to the running sums (ring slot r mod 5).
    auto accum = [&](int s, int r) {
        const uint64_t* rowB = sB + s * (kStageB / 8) + r * kRowB;
        const uint64_t* rowM = sM + s * (kStageM / 8) + r * kRowM;
        uint2 bw[kCPT], mw[NWD];
        const uint4 q0 = *reinterpret_cast<const uint4*>(rowB + boff[0]);
        const uint4 q1 = *reinterpret_cast<const uint4*>(rowB + boff[1]);
        bw[0] = make_uint2(q0.x, q0.y); bw[1] = make_uint2(q0.z, q0.w);
        bw[2] = make_uint2(q1.x, q1.y); bw[3] = make_uint2(q1.z, q1.w);
#pragma unroll
        for (int k = 0; k < NWD / 2; ++k) {
            const uint4 q = *reinterpret_cast<const uint4*>(rowM + moff[k]);
            mw[2 * k] = make_uint2(q.x, q.y);
            mw[2 * k + 1] = make_uint2(q.z, q.w);
        }
        const int slot = r % kRB;
#pragma unroll
        for (int c = 0; c < kCPT; ++c)
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                // left-to-right: column x - d sits at mw[c - j + DPW]; right-to-left: x + d at mw[c + j]
                const int k0 = DIR == 0 ? c - 2 * p + DPW : c + 2 * p;
                const int k1 = DIR == 0 ? c - 2 * p - 1 + DPW : c + 2 * p + 1;
                const uint32_t e0 = __popc(bw[c].x ^ mw[k0].x) + __popc(bw[c].y ^ mw[k0].y);
                const uint32_t e1 = __popc(bw[c].x ^ mw[k1].x) + __popc(bw[c].y ^ mw[k1].y);
                const uint32_t P = e0 + (e1 << 16);
                V[c][p] = V[c][p] + P - ring[slot][c][p];
                ring[slot][c][p] = P;
            }
    };

    // Writes this thread's curve codes of output row oy (see MatchArgs): one
    // 32-bit word (4 disparities) per column and disparity group, the 4
    // columns of a lane as one 16-byte store (word index xs + 4 lane + 2 is a
    // multiple of 4); lanes 0 and 31 skip their halo columns. The stores are
    // streaming (st.global.cs, evict-first): the volume is written once and
    // is larger than L2, and letting it settle there evicted the descriptor
    // rows the next strips read (0.286 -> 0.251 ms for census + L->R +
    // curves at 1080p, D = 128).
    auto store_curve = [&](const uint32_t (&C)[kCPT][NP], int oy) {
        const int y = y0 + oy;
        constexpr int NG = DPW / 4;
        uint32_t wv[kCPT][NG];
#pragma unroll
        for (int c = 0; c < kCPT; ++c) {
#pragma unroll
            for (int q = 0; q < NG; ++q) {
                // C < 2048 per 16-bit half, so byte 0 and byte 2 of C >> 3 are
                // the two codes (bits of the high half shifted into byte 1 are
                // never selected)
                uint32_t w = __byte_perm(C[c][2 * q] >> 3, C[c][2 * q + 1] >> 3, 0x6420);
                if (EDGE) {  // disparities above lim[c] read 255
                    const int nvalid = min(max(lim[c] - (dw + 4 * q) + 1, 0), 4);
                    w |= nvalid >= 4 ? 0u : (0xFFFFFFFFu << (8 * nvalid));
                }
                wv[c][q] = w;
            }
        }
#pragma unroll
        for (int q = 0; q < NG; ++q) {
            const int g = (dw >> 2) + q;
            if (g >= a.curve_groups) break;
            uint32_t* dst = a.curve + ((size_t)y * a.curve_groups + g) * a.curve_pitch + (xs + 4 * lane + 2);
            if (xs + kTWV - kAR <= a.W) {  // warp-uniform: every own column is inside the image
                // lanes 1..30 store 4 columns; lane 0 its columns 2, 3; lane 31 its columns 0, 1
                if (lane > 0 && lane < 31) {
                    __stcs(reinterpret_cast<uint4*>(dst), make_uint4(wv[0][q], wv[1][q], wv[2][q], wv[3][q]));
                } else {
                    const bool l0 = lane == 0;
                    __stcs(reinterpret_cast<uint2*>(dst + (l0 ? 2 : 0)),
                           l0 ? make_uint2(wv[2][q], wv[3][q]) : make_uint2(wv[0][q], wv[1][q]));
                }
            } else {
#pragma unroll
                for (int c = 0; c < kCPT; ++c) {
                    const int v = 4 * lane + c;
                    if (v >= kAR && v < kAR + kTWO && xs + v < a.W) __stcs(&dst[c], wv[c][q]);
                }
            }
        }
    };

    // Horizontal 5-wide sums of V and winner-take-all of this thread's
    // disparities for its 4 columns, merged into key buffer `buf`, slot r
    // (output row oy of the strip).
    // Keys are stored column-interleaved (index c * 32 + lane) so the 32 lanes'
    // atomics hit 32 different banks; the halo columns' slots (V columns 0, 1,
    // 126, 127) receive values nobody reads.
    auto emit = [&](int buf, int r, int oy) {
        uint32_t C[kCPT][NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const uint32_t h0 = __shfl_up_sync(0xffffffffu, V[2][p], 1);
            const uint32_t h1 = __shfl_up_sync(0xffffffffu, V[3][p], 1);
            const uint32_t h4 = __shfl_down_sync(0xffffffffu, V[0][p], 1);
            const uint32_t h5 = __shfl_down_sync(0xffffffffu, V[1][p], 1);
            C[0][p] = h0 + h1 + V[0][p] + V[1][p] + V[2][p];
            C[1][p] = C[0][p] + V[3][p] - h0;
            C[2][p] = C[1][p] + h4 - h1;
            C[3][p] = C[2][p] + h5 - V[0][p];
        }
        if constexpr (CURVE) {
            if (oy >= 0 && oy < rows_here) store_curve(C, oy);
        }
        uint32_t* krow = sKey + ((buf * kGroups + grp) * kBR + r) * kTWV + lane;
        // 16-bit keys C << 5 | (d & 31) of (column c, relative disparities
        // dw + 2p, dw + 2p + 1) in the halves of kk[c][p]
        uint32_t kk[kCPT][NP];
#pragma unroll
        for (int c = 0; c < kCPT; ++c) {
            uint32_t* k = kk[c];
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                k[p] = (C[c][p] << 5) + dconst[p];
                if (EDGE) {
                    const int dlo = dw + 2 * p;
                    k[p] |= (dlo > lim[c] || dlo < a.dfirst ? 0x0000FFFFu : 0u) |
                            (dlo + 1 > lim[c] ? 0xFFFF0000u : 0u);
                }
                // columns that may not bid for the right view (not outputs of
                // this pass either, so their left-to-right keys do not matter)
                if constexpr (RL) k[p] |= rlbad[c];
            }
            uint32_t m;
            if (NP == 4) {
                m = dev::min3_u16x2(k[0], k[1], k[NP > 2 ? 2 : 0]);
                m = dev::min_u16x2(m, k[NP > 3 ? 3 : 0]);
            } else {
                m = dev::min_u16x2(k[0], k[NP > 1 ? 1 : 0]);
            }
            m = dev::min_u16x2(m, __byte_perm(m, 0u, 0x1032));  // both halves = the minimum
            atomicMin(&krow[c * 32], m);
        }
        if constexpr (RL) {
            // Cost of (column c, relative disparity dw + j) bids for right
            // pixel index c - j + base: min along each anti-diagonal
            // ad = c - j, one shared atomic each, on the same 16-bit keys.
            // Word kk[c][p] holds diagonals c - 2p (low half) and c - 2p - 1
            // (high half); M[a] = min over the words with c - 2p = a, so
            // diagonal ad = min(low half of M[ad], high half of M[ad + 1]):
            // one shift and one packed min put it in a high half.
            constexpr int A0 = -(DPW - 2), A1 = kCPT - 1;
            uint32_t M[A1 - A0 + 1];
#pragma unroll
            for (int q = 0; q <= A1 - A0; ++q) {
                bool first = true;
#pragma unroll
                for (int c = 0; c < kCPT; ++c)
#pragma unroll
                    for (int p = 0; p < NP; ++p)
                        if (c - 2 * p == q + A0) {
                            M[q] = first ? kk[c][p] : dev::min_u16x2(M[q], kk[c][p]);
                            first = false;
                        }
            }
            // right-view index i = 4 * lane + (kDPC - 1) - (dw - dz0) + ad;
            // (kDPC - 1) - (dw - dz0) = 4 q + 3 (dw - dz0 a multiple of 4), so
            // word(i) = ((3 + ad) & 3) * kRLQ + lane + q + ((3 + ad) >> 2).
            // Slot values: the key in the high half (the low half only
            // orders equal keys and is never read).
            uint32_t* rrow =
                sKeyRL + ((buf * kGroups + grp) * kBR + r) * kRLW + lane + ((kDPC - 1 - (dw - dz0)) >> 2);
#pragma unroll
            for (int ad = A0 - 1; ad <= A1; ++ad) {
                uint32_t z;
                if (ad == A0 - 1) z = M[0];
                else if (ad == A1) z = M[A1 - A0] << 16;
                else z = dev::min_u16x2(M[ad - A0] << 16, M[ad + 1 - A0]);
                atomicMin(&rrow[((3 + ad) & 3) * kRLQ + ((3 + ad) >> 2)], z);
            }
        }
    };

    // Merges the groups of key buffer `buf`, slots r0 .. r1-1 (output row
    // oy0 + slot), writes or forwards the result, and resets the slots.
    auto flush = [&](int buf, int oy0, int r0, int r1) {
        for (int idx = tid; idx < (r1 - r0) * kTWO; idx += NT) {
            const int r = r0 + idx / kTWO, ox = idx % kTWO;
            const int v = ox + kAR;                      // V column
            const int slot = (v & 3) * 32 + (v >> 2);    // column-interleaved key index
            uint32_t best = 0xFFFFFFFFu;
#pragma unroll
            for (int g = 0; g < kGroups; ++g) {
                uint32_t* kp = sKey + ((buf * kGroups + g) * kBR + r) * kTWV + slot;
                const uint32_t k16 = *kp & 0xFFFFu;
                *kp = 0xFFFFFFFFu;
                const uint32_t key = ((k16 & 0xFFE0u) << 11) | ((k16 & 31u) + uint32_t(dz0 + 32 * g));
                best = min(best, key);
            }
            const int oy = oy0 + r, x = xs + v, y = y0 + oy;
            if (oy >= 0 && oy < rows_here && x < a.W) {
                if (t.nbz == 1) {
                    const bool valid = x >= kAR && x < a.W - kAR && y >= kAR && y < a.H - kAR;
                    store_disp(a.out, a.out_pitch, a.out_type, x, y, valid, best, a.dmin);
                } else if (a.merge_last) {
                    a.keys[(size_t)t.bz * a.W * a.H + (size_t)y * a.W + x] = best;
                } else {
                    atomicMin(&a.keys[(size_t)y * a.W + x], best);
                }
            }
        }
    };
    // The fused right-to-left keys of buffer `buf`, slots r0 .. r1-1: bids
    // into the global plane, slots reset.
    auto flush_rl = [&](int buf, int oy0, int r0, int r1) {
        if constexpr (RL) {
            const int xr0 = xs - a.dmin - dz0 - (kDPC - 1);  // right-view column of index 0
            for (int idx = tid; idx < (r1 - r0) * kRLW; idx += NT) {
                const int r = r0 + idx / kRLW, i = idx % kRLW;
                uint32_t best = 0xFFFFFFFFu;
#pragma unroll
                for (int g = 0; g < kGroups; ++g) {
                    uint32_t* kp = sKeyRL + ((buf * kGroups + g) * kBR + r) * kRLW + rl_word(i);
                    const uint32_t k16 = *kp >> 16;
                    *kp = 0xFFFFFFFFu;
                    if (k16 < (2047u << 5))  // a cost below 2047
                        best = min(best, ((k16 >> 5) << 16) | (uint32_t(a.dmin + dz0 + 32 * g) + (k16 & 31u)));
                }
                const int oy = oy0 + r, x = xr0 + i, y = y0 + oy;
                if (best != 0xFFFFFFFFu && oy >= 0 && oy < rows_here && x >= 0 && x < a.W)
                    atomicMin(&a.rl_keys[(size_t)y * a.rl_pitch + x], best | a.rl_tag);
            }
        }
    };
    unsigned* group_counter = reinterpret_cast<unsigned*>(a.counters ? &a.counters[t.by * t.nbx + t.bx] : nullptr);

    // Cost row i = kBR * b + r. Before row i is added, V holds rows i-5..i-1:
    // the window of output row i - 5, whose keys go to buffer b & 1, slot r.
    // Stage s is used by batches s, s + 2, ...: its (b >> 1)-th use in this
    // tile completes phase par[s] + (b >> 1) of its mbarrier.
    for (int b = 0; b < nb; ++b) {
        const int s = b & 1;
        if (!dev::mbar_wait_bounded(&bars[s], (par[s] + (b >> 1)) & 1)) *sflag = 1;
        if (warp_active) {
            if (b == 0) {
#pragma unroll
                for (int r = 0; r < kBR; ++r) {
                    if (r >= kRB) emit(0, r, r - kRB);
                    accum(s, r);
                }
            } else {
#pragma unroll
                for (int r = 0; r < kBR; ++r) {
                    emit(b & 1, r, kBR * b - kRB + r);
                    accum(s, r);
                }
            }
        }
        __syncthreads();  // stage s consumed; key buffer b & 1 complete
        if (*sflag) {     // a tile load never arrived: report and leave together
            if (tid == 0) {
                dev::report(a.status, CT_ETIMEOUT);
                if (b + 1 < nb) dev::mbar_wait_bounded(&bars[s ^ 1], (par[s ^ 1] + ((b + 1) >> 1)) & 1);
                if (t.nbz > 1 && a.merge_last) {  // keep the group counter consistent
                    if (atomicAdd(group_counter, 1u) == unsigned(t.nbz) - 1) *group_counter = 0u;
                }
            }
            return TileResult{false, true};
        }
        if (tid == 0 && b + 2 < nb) {
            dev::fence_proxy_async();
            dev::mbar_arrive_expect_tx(&bars[s], kBytes);
            dev::tma_load_4d(sB + s * (kStageB / 8), tmB, 0, i0, 0, ye0 + (b + 2) * kBR, &bars[s]);
            dev::tma_load_4d(sM + s * (kStageM / 8), tmM, 0, j0, 0, ye0 + (b + 2) * kBR, &bars[s]);
        }
        flush(b & 1, kBR * b - kRB, b == 0 ? kRB : 0, kBR);
        flush_rl(b & 1, kBR * b - kRB, b == 0 ? kRB : 0, kBR);
    }
    // the window ending at the last staged row: output kBR * nb - 5, buffer nb & 1, slot 0
    if (warp_active) emit(nb & 1, 0, kBR * nb - kRB);
    __syncthreads();
    flush(nb & 1, kBR * nb - kRB, 0, 1);
    flush_rl(nb & 1, kBR * nb - kRB, 0, 1);

    if (t.nbz == 1) return TileResult{true, false};
    if (!a.merge_last) return TileResult{false, false};
    // The last CTA of this (strip, column tile) group merges the groups' key
    // planes. Writers fence before counting; the merger fences after.
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(group_counter, 1u);
        sflag[1] = prev == unsigned(t.nbz) - 1;
        if (sflag[1]) *group_counter = 0u;  // ready for the next call
    }
    __syncthreads();
    const bool last = sflag[1] != 0;
    if (last) {
        __threadfence();
        const size_t plane = (size_t)a.W * a.H;
        for (int idx = tid; idx < rows_here * kTWO; idx += NT) {
            const int oy = idx / kTWO, x = xs + kAR + idx % kTWO, y = y0 + oy;
            if (x >= a.W) continue;
            const uint32_t* kp = a.keys + (size_t)y * a.W + x;
            uint32_t best = 0xFFFFFFFFu;
            for (int z = 0; z < t.nbz; ++z) best = min(best, __ldcg(kp + z * plane));
            const bool valid = x >= kAR && x < a.W - kAR && y >= kAR && y < a.H - kAR;
            store_disp(a.out, a.out_pitch, a.out_type, x, y, valid, best, a.dmin);
        }
    }
    return TileResult{last, false};
}

// Shared-memory carve-up common to the single-image and the batched kernels.
struct Smem {
    uint64_t* sB;     // [2 stages][kBR][2][kPB][2]
    uint64_t* sM;     // [2 stages][kBR][2][kPM][2]
    uint32_t* sKey;   // [2][kGroups][kBR][kTWV]
    uint64_t* bars;   // [2]
    int* sflag;       // [4]
    uint32_t* sKeyRL; // [2][kGroups][kBR][kRLW] (kernels with the fused right-to-left keys only)
    __device__ explicit Smem(unsigned char* raw)
        : sB(reinterpret_cast<uint64_t*>(raw)),
          sM(reinterpret_cast<uint64_t*>(raw + 2 * kStageB)),
          sKey(reinterpret_cast<uint32_t*>(raw + 2 * (kStageB + kStageM))),
          bars(reinterpret_cast<uint64_t*>(raw + 2 * (kStageB + kStageM) + size_t(2) * kGroups * kBR * kTWV * 4)),
          sflag(reinterpret_cast<int*>(bars + 2)),
          sKeyRL(reinterpret_cast<uint32_t*>(raw + rl_offset())) {}
};

// Runs one tile. The mbarriers must be initialised; par[s] counts the phases
// stage s has completed so far in this CTA and is advanced here.
template <int DIR, int DPW, bool CURVE = false, bool RL = false>
__device__ TileResult run_tile(const CUtensorMap* tmB, const CUtensorMap* tmM, const MatchArgs& a, const Tile& t,
                               const Smem& sm, uint32_t* par) {
    const int tid = threadIdx.x;
    const int xs = t.bx * kTWO - kAR;             // first V column
    const int y0 = t.by * a.th;                   // first output row
    const int ye0 = y0 - kAR;                     // first cost row
    const int dz0 = t.bz * kDPC;
    // first staged match column (even: xs, dz0, kDPC and dmin are)
    const int ms = DIR == 0 ? xs - a.dmin - dz0 - kDPC : xs + a.dmin + dz0;
    const int rows_here = min(a.th, a.H - y0);
    const int nb = (rows_here + 2 * kAR + kBR - 1) / kBR;   // batches of 10 cost rows
    const bool interior = (dz0 + kDPC <= a.D) && !(a.dfirst > 0 && dz0 == 0) &&
                          (DIR == 0 ? (xs - a.dmin >= dz0 + kDPC - 1)
                                    : (xs + a.dmin + dz0 + kDPC - 1 + kTWV <= a.W));

    if (tid == 0) {
        dev::prefetch_tmap(tmB);
        dev::prefetch_tmap(tmM);
        sm.sflag[0] = 0;
    }
    for (int i = tid; i < 2 * kGroups * kBR * kTWV; i += Var<DPW>::kNT) sm.sKey[i] = 0xFFFFFFFFu;
    if constexpr (RL)
        for (int i = tid; i < 2 * kGroups * kBR * kRLW; i += Var<DPW>::kNT) sm.sKeyRL[i] = 0xFFFFFFFFu;
    __syncthreads();
    if (tid == 0) {
        for (int b = 0; b < 2 && b < nb; ++b) {
            dev::fence_proxy_async();
            dev::mbar_arrive_expect_tx(&sm.bars[b], kTxB + kTxM);
            dev::tma_load_4d(sm.sB + b * (kStageB / 8), tmB, 0, (xs >> 1) >> 1, 0, ye0 + b * kBR, &sm.bars[b]);
            dev::tma_load_4d(sm.sM + b * (kStageM / 8), tmM, 0, (ms >> 1) >> 1, 0, ye0 + b * kBR, &sm.bars[b]);
        }
    }
    const TileResult res =
        interior ? match_body<DIR, false, DPW, CURVE, RL>(tmB, tmM, a, t, sm.sB, sm.sM, sm.sKey, sm.bars, sm.sflag,
                                                          par, nb, rows_here, xs, y0, ye0, dz0, ms, sm.sKeyRL)
                 : match_body<DIR, true, DPW, CURVE, RL>(tmB, tmM, a, t, sm.sB, sm.sM, sm.sKey, sm.bars, sm.sflag,
                                                         par, nb, rows_here, xs, y0, ye0, dz0, ms, sm.sKeyRL);
    par[0] += (nb + 1) / 2;
    par[1] += nb / 2;
    __syncthreads();  // the next tile reuses the shared memory
    return res;
}

__device__ __forceinline__ void init_barriers(const Smem& sm) {
    if (threadIdx.x == 0) {
        dev::mbar_init(&sm.bars[0], 1);
        dev::mbar_init(&sm.bars[1], 1);
        dev::fence_barrier_init();
    }
    __syncthreads();
}

template <int DIR, int DPW, bool CURVE = false, bool RL = false>
__global__ void __launch_bounds__(Var<DPW>::kNT, 1)
    census_match_kernel(const __grid_constant__ CUtensorMap tmB, const __grid_constant__ CUtensorMap tmM,
                        MatchArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const Smem sm(smem_raw);
    // A kernel launched after this one with programmatic stream
    // serialisation (the other direction, the cross-check, the
    // confidence-net inference) may be scheduled once every CTA of this grid
    // has started; it waits for this grid's results itself
    // (griddepcontrol.wait). Without such a launch this is a no-op.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    init_barriers(sm);
    // This launch is itself programmatic: the previous kernel (census or the
    // other direction) must be complete before any global read or write.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    uint32_t par[2] = {0, 0};
    const Tile t{int(blockIdx.x), int(blockIdx.y), int(blockIdx.z), int(gridDim.x), int(gridDim.z)};
    run_tile<DIR, DPW, CURVE, RL>(&tmB, &tmM, a, t, sm, par);
}

// Map code of a right-view key of the fused pass (what store_disp writes
// for it): a disparity iff the key carries this call's tag, a cost below
// 2047 and the pixel is inside the border.
template <typename T>
__device__ __forceinline__ T rl_code(uint32_t key, uint32_t tag, bool inside) {
    const bool ok = inside && (key & (0x1Fu << kRLTagShift)) == tag && ((key >> 16) & 0x7FFu) < 2047u;
    const uint32_t d = key & 0xFFFFu;
    if constexpr (sizeof(T) == 1) return ok ? T(d) : T(0xFF);
    else return ok ? T(d + 1) : T(0xFFFF);
}
// Disparity of a map code (the cross-check's reading: U8 0xFF and U16
// codes outside CT_DISP_FIRST .. CT_DISP_LAST are not disparities).
template <typename T>
__device__ __forceinline__ bool map_disp(T v, int& d) {
    if constexpr (sizeof(T) == 1) {
        d = v;
        return v != 0xFF;
    } else {
        d = int(v) - 1;
        return v >= CT_DISP_FIRST && v <= CT_DISP_LAST;
    }
}

// After the fused pass, one thread per 16 bytes of a map row (16 U8 or 8 U16
// pixels): writes the right-view map from the keys of this call (rl_out, when
// given) and the left-to-right cross-check of the left map lr (ck_out, when
// given): a left disparity d at x is kept iff the right view's code at x - d
// confirms it as crosscheck_kernel reads the right-view map (U16: the codes
// within tol; U8: a disparity within tol), from the keys directly. The keys
// stay in place.
template <typename T>
__global__ void __launch_bounds__(128) rl_check_kernel(const uint32_t* keys, size_t kpitch, uint32_t tag, int W,
                                                       int H, int r, T* rl_out, size_t rl_pitch_b, const T* lr,
                                                       size_t lr_pitch_b, T* ck_out, size_t ck_pitch_b, int tol) {
    constexpr int PX = 16 / sizeof(T);
    // launched with programmatic stream serialisation after the matcher
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int x0 = (blockIdx.x * blockDim.x + threadIdx.x) * PX;
    const int y = blockIdx.y;
    if (x0 >= W) return;
    const uint32_t* krow = keys + (size_t)y * kpitch;
    const bool yin = y >= r && y < H - r;
    const bool full = x0 + PX <= W;  // map rows are 16-byte aligned, x0 a multiple of PX
    union Px {
        uint4 q;
        T v[PX];
    };
    if (rl_out) {
        T* orow = reinterpret_cast<T*>(reinterpret_cast<char*>(rl_out) + (size_t)y * rl_pitch_b);
        Px o;
#pragma unroll
        for (int q = 0; q < PX / 4; ++q) {
            // key rows are 16-byte aligned with a multiple of 4 words
            uint4 k4 = make_uint4(~0u, ~0u, ~0u, ~0u);
            if (x0 + 4 * q < W) k4 = *reinterpret_cast<const uint4*>(krow + x0 + 4 * q);
            const uint32_t kk[4] = {k4.x, k4.y, k4.z, k4.w};
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int x = x0 + 4 * q + i;
                o.v[4 * q + i] = rl_code<T>(kk[i], tag, yin && x >= r && x < W - r);
            }
        }
        if (full) *reinterpret_cast<uint4*>(orow + x0) = o.q;
        else
            for (int i = 0; i < PX; ++i)
                if (x0 + i < W) orow[x0 + i] = o.v[i];
    }
    if (ck_out) {
        const T* brow = reinterpret_cast<const T*>(reinterpret_cast<const char*>(lr) + (size_t)y * lr_pitch_b);
        T* crow = reinterpret_cast<T*>(reinterpret_cast<char*>(ck_out) + (size_t)y * ck_pitch_b);
        Px in, res;
        if (full) in.q = *reinterpret_cast<const uint4*>(brow + x0);
        else
            for (int i = 0; i < PX; ++i) in.v[i] = x0 + i < W ? brow[x0 + i] : T(0);
#pragma unroll
        for (int i = 0; i < PX; ++i) {
            const int x = x0 + i;
            const T v = in.v[i];
            T out = v;
            int d;
            if (map_disp<T>(v, d)) {
                const int xo = x - d;
                out = sizeof(T) == 1 ? T(0xFF) : T(CT_DISP_INCONSISTENT);
                if (xo >= 0 && xo < W) {
                    const T vo = rl_code<T>(__ldg(krow + xo), tag, yin && xo >= r && xo < W - r);
                    int dd;
                    // U16: raw codes compared (CrossCheckDisparityMaps.cu:94);
                    // U8: only a disparity confirms
                    const bool ok = sizeof(T) == 2 ? abs(int(vo) - int(v)) <= tol
                                                   : map_disp<T>(vo, dd) && abs(dd - d) <= tol;
                    if (ok) out = v;
                }
            }
            res.v[i] = out;
        }
        if (full) *reinterpret_cast<uint4*>(crow + x0) = res.q;
        else
            for (int i = 0; i < PX; ++i)
                if (x0 + i < W) crow[x0 + i] = res.v[i];
    }
}

// Converts merged keys to disparities and resets the keys for the next call.
// (static: each translation unit that launches it has its own copy.)
static __global__ void keys_finalize_kernel(uint32_t* keys, int W, int H, int r, void* out, size_t out_pitch,
                                            int out_type, int dmin) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    uint32_t* kp = &keys[(size_t)y * W + x];
    const uint32_t key = *kp;
    *kp = 0xFFFFFFFFu;
    const bool valid = x >= r && x < W - r && y >= r && y < H - r;
    store_disp(out, out_pitch, out_type, x, y, valid, key, dmin);
}

// Strip height: picks the height that minimises (waves of CTAs over the SMs)
// x (cost rows per CTA), i.e. the trade-off between the 4 halo rows every
// strip recomputes and the tail of the last wave (one CTA per SM). Heights
// with th + 4 a multiple of 10 waste no staged rows.
inline int pick_strip_height(int W, int H, int D, int sms) {
    const int tiles = ((W + kTWO - 1) / kTWO) * ((D + kDPC - 1) / kDPC);
    int best = 36;
    long best_cost = -1;
    for (int th = 16; th <= 506; th += kBR) {
        const int strips = (H + th - 1) / th;
        const long ctas = long(strips) * tiles;
        const long waves = (ctas + sms - 1) / sms;
        const int rows = min(th, H);
        const long cost = waves * long((rows + 2 * kAR + kBR - 1) / kBR * kBR);
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = th;
        }
    }
    return best;
}

// 4D TMA maps over pair-planar descriptor buffers (dims: word in pair, pair
// index, plane, row): `tb` stages base rows (kPB pairs per plane), `tm` match
// rows (kPM), kBR rows per box.
inline int make_planar_maps(CUtensorMap* tb, CUtensorMap* tm, const uint64_t* base, const uint64_t* match, int W,
                            int H) {
    const uint64_t ni = uint64_t(planar_ni(W));
    const uint64_t dims[4] = {2, ni, 2, uint64_t(H)};
    const uint64_t strides[3] = {16, ni * 16, ni * 32};
    const uint32_t box_b[4] = {2, kPB, 2, kBR}, box_m[4] = {2, kPM, 2, kBR};
    if (int rc = ct::make_tmap_nd(tb, base, CU_TENSOR_MAP_DATA_TYPE_UINT64, 8, 4, dims, strides, box_b)) return rc;
    return ct::make_tmap_nd(tm, match, CU_TENSOR_MAP_DATA_TYPE_UINT64, 8, 4, dims, strides, box_m);
}

// Allows the 71 KB of dynamic shared memory on the current device for every
// kernel instantiation. Sets function attributes only (no allocation).
inline cudaError_t prepare_census_match() {
    const int smem = int(smem_bytes());
    const void* kernels[] = {
        reinterpret_cast<const void*>(census_match_kernel<0, 4>), reinterpret_cast<const void*>(census_match_kernel<0, 8>),
        reinterpret_cast<const void*>(census_match_kernel<1, 4>), reinterpret_cast<const void*>(census_match_kernel<1, 8>),
        reinterpret_cast<const void*>(census_match_kernel<0, 4, true>),
        reinterpret_cast<const void*>(census_match_kernel<0, 8, true>),
        reinterpret_cast<const void*>(census_match_kernel<1, 4, true>),
        reinterpret_cast<const void*>(census_match_kernel<1, 8, true>)};
    for (const void* k : kernels) {
        const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
    }
    const void* fused[] = {reinterpret_cast<const void*>(census_match_kernel<0, 4, false, true>),
                           reinterpret_cast<const void*>(census_match_kernel<0, 8, false, true>)};
    for (const void* k : fused) {
        const cudaError_t e =
            cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_bytes_rl()));
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Launches one matching pass (+ the key finalize when D is split over CTAs).
template <int DIR>
inline cudaError_t launch_census_match(const CUtensorMap& tb, const CUtensorMap& tm, const MatchArgs& a,
                                       cudaStream_t s, int dpw = 4) {
    dim3 grid((a.W + kTWO - 1) / kTWO, (a.H + a.th - 1) / a.th, (a.D + kDPC - 1) / kDPC);
    // programmatic stream serialisation: the launch overlaps the previous
    // kernel's tail; the kernel waits (griddepcontrol.wait) before reading
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(dpw == 8 ? Var<8>::kNT : Var<4>::kNT);
    cfg.dynamicSmemBytes = smem_bytes();
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e;
    if (DIR == 0 && a.rl_keys) {
        cfg.dynamicSmemBytes = smem_bytes_rl();
        e = dpw == 8 ? cudaLaunchKernelEx(&cfg, census_match_kernel<0, 8, false, true>, tb, tm, a)
                     : cudaLaunchKernelEx(&cfg, census_match_kernel<0, 4, false, true>, tb, tm, a);
    } else if (a.curve)
        e = dpw == 8 ? cudaLaunchKernelEx(&cfg, census_match_kernel<DIR, 8, true>, tb, tm, a)
                     : cudaLaunchKernelEx(&cfg, census_match_kernel<DIR, 4, true>, tb, tm, a);
    else
        e = dpw == 8 ? cudaLaunchKernelEx(&cfg, census_match_kernel<DIR, 8, false>, tb, tm, a)
                     : cudaLaunchKernelEx(&cfg, census_match_kernel<DIR, 4, false>, tb, tm, a);
    if (e != cudaSuccess) return e;
    e = cudaGetLastError();
    if (e != cudaSuccess || grid.z == 1 || a.merge_last) return e;
    keys_finalize_kernel<<<dim3((a.W + 255) / 256, a.H), 256, 0, s>>>(a.keys, a.W, a.H, kAR, a.out, a.out_pitch,
                                                                      a.out_type, a.dmin);
    return cudaGetLastError();
}

}  // namespace cm
}  // namespace ct
