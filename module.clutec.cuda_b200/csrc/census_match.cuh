// census_match.cuh — census transform and the fused census matcher kernel:
// Hamming cost (popcount of XOR of 64-bit descriptors) + 5x5 box aggregation
// + winner-take-all, one launch per direction.
//
// Mapping to B200:
//  * A CTA owns a tile of 128 "V columns" (124 output columns plus 2 halo
//    columns on each side) x th output rows x 64 disparities. Its 8 warps share
//    the same columns and rows; warp w owns disparities dz0 + 8w .. +7 and
//    lane L owns the 4 adjacent columns 4L..4L+3.
//  * Descriptor rows are staged in shared memory by 2D TMA tile loads (one box
//    of 5 rows of the base image and one of the match image per batch), two
//    batches in flight, completion tracked by mbarriers with bounded waits.
//  * Each thread keeps, in registers, the vertical running sums V of its 4
//    columns x 8 disparities and a 5-deep ring of the per-row Hamming costs
//    (the role of AlgoArraySum_W32H16::SumCache's vertical pass,
//    Kernel.Algo.ArraySum_W32H16.h:163-182). Costs for two disparities are
//    packed in the two 16-bit halves of one register, so every add/sub of the
//    running sums handles two disparities.
//  * The horizontal pass (ArraySum_W32H16.h:186-200) takes the 2 halo columns
//    from the neighbouring lanes with warp shuffles and runs a 5-wide running
//    sum over the thread's columns.
//  * Winner-take-all folds the disparity into the low 5 bits of each 16-bit
//    lane (key = C << 5 | d mod 32, C <= 25 * 63 = 1575 so it fits), so the min
//    over 8 disparities is two packed 3-way mins, and the lowest d wins ties
//    by construction (the reference's strict '<' scanning d upward). Warps
//    merge per pixel through a shared-memory atomicMin on (C << 16 | d); CTAs
//    that split D merge through a global atomicMin.
#pragma once

#include <cstdint>

#include "ct_device.cuh"

namespace ct {
namespace cm {

constexpr int kCPT = 4;                 // columns per thread
constexpr int kTWV = 32 * kCPT;         // 128 V columns per tile
constexpr int kAR = 2;                  // aggregation radius (5x5)
constexpr int kTWO = kTWV - 2 * kAR;    // 124 output columns per tile
constexpr int kDPW = 8;                 // disparities per warp
constexpr int kNW = 8;                  // warps per CTA
constexpr int kNT = kNW * 32;           // threads per CTA
constexpr int kDPC = kDPW * kNW;        // 64 disparities per CTA
constexpr int kRB = 2 * kAR + 1;        // rows per TMA batch = ring depth = 5
constexpr int kMW = kTWV + kDPC;        // 192 match columns staged per row

// Output rows per CTA: th + 2*kAR must be a multiple of kRB.
__host__ __device__ constexpr bool valid_th(int th) { return th > 0 && (th + 2 * kAR) % kRB == 0; }

struct MatchArgs {
    int W, H, D;
    int th;             // output rows per CTA
    int nbatch;         // (th + 2*kAR) / kRB
    uint32_t* keys;     // W*H keys merged by atomicMin when gridDim.z > 1
    void* out;          // direct disparity output when gridDim.z == 1
    size_t out_pitch;
    int out_type;       // CT_PIX_U8 / CT_PIX_U16
    int32_t* status;
};

__host__ __device__ constexpr size_t smem_bytes(int th) {
    return size_t(2) * kRB * kTWV * 8 + size_t(2) * kRB * kMW * 8 + size_t(th) * kTWO * 4 + 2 * 8;
}

// Disparity code for an output pixel from its merged key.
__device__ __forceinline__ void store_disp(void* out, size_t pitch, int type, int x, int y, bool valid,
                                           uint32_t key) {
    const uint32_t d = key & 0xFFFFu;
    const bool ok = valid && (key >> 16) < 2047u;
    if (type == 1) {  // CT_PIX_U8
        reinterpret_cast<uint8_t*>(static_cast<char*>(out) + (size_t)y * pitch)[x] = ok ? uint8_t(d) : uint8_t(0xFF);
    } else {  // CT_PIX_U16 (EDisparityId)
        reinterpret_cast<uint16_t*>(static_cast<char*>(out) + (size_t)y * pitch)[x] =
            ok ? uint16_t(d + 1) : uint16_t(0xFFFF);
    }
}

template <int DIR>
__global__ void __launch_bounds__(kNT, 1)
    census_match_kernel(const __grid_constant__ CUtensorMap tmB, const __grid_constant__ CUtensorMap tmM,
                        MatchArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t* sB = reinterpret_cast<uint64_t*>(smem_raw);   // [2][kRB][kTWV]
    uint64_t* sM = sB + 2 * kRB * kTWV;                      // [2][kRB][kMW]
    uint32_t* sKey = reinterpret_cast<uint32_t*>(sM + 2 * kRB * kMW);  // [th][kTWO]
    uint64_t* bars = reinterpret_cast<uint64_t*>(sKey + a.th * kTWO);  // [2]

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int xs = blockIdx.x * kTWO - kAR;       // first V column
    const int y0 = blockIdx.y * a.th;             // first output row
    const int ye0 = y0 - kAR;                     // first cost row
    const int dz0 = blockIdx.z * kDPC;
    const int dw = dz0 + warp * kDPW;
    const int ms = DIR == 0 ? xs - dz0 - kDPC : xs + dz0;  // first staged match column
    const bool warp_active = dw < a.D;
    const bool interior = (dz0 + kDPC <= a.D) &&
                          (DIR == 0 ? (xs >= dz0 + kDPC - 1) : (xs + dz0 + kDPC - 1 + kTWV <= a.W));

    constexpr uint32_t kBytesB = kRB * kTWV * 8, kBytesM = kRB * kMW * 8;

    if (tid == 0) {
        dev::prefetch_tmap(&tmB);
        dev::prefetch_tmap(&tmM);
        dev::mbar_init(&bars[0], 1);
        dev::mbar_init(&bars[1], 1);
        dev::fence_barrier_init();
    }
    for (int i = tid; i < a.th * kTWO; i += kNT) sKey[i] = 0xFFFFFFFFu;
    __syncthreads();
    if (tid == 0) {
        for (int b = 0; b < 2 && b < a.nbatch; ++b) {
            dev::mbar_arrive_expect_tx(&bars[b], kBytesB + kBytesM);
            dev::tma_load_2d(sB + b * kRB * kTWV, &tmB, xs, ye0 + b * kRB, &bars[b]);
            dev::tma_load_2d(sM + b * kRB * kMW, &tmM, ms, ye0 + b * kRB, &bars[b]);
        }
    }

    // Per-thread state: running vertical sums and the ring of packed costs.
    uint32_t V[kCPT][4];
    uint32_t ring[kRB][kCPT][4];
#pragma unroll
    for (int c = 0; c < kCPT; ++c)
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            V[c][p] = 0;
#pragma unroll
            for (int r = 0; r < kRB; ++r) ring[r][c][p] = 0;
        }
    // d mod 32 of the two disparities of each pair, packed.
    uint32_t dconst[4];
#pragma unroll
    for (int p = 0; p < 4; ++p)
        dconst[p] = uint32_t((dw + 2 * p) & 31) | (uint32_t((dw + 2 * p + 1) & 31) << 16);
    const uint32_t dgroup = uint32_t(dw & ~31);
    const int mstart = DIR == 0 ? 4 * lane + kDPC - 8 - kDPW * warp : 4 * lane + kDPW * warp;

    for (int b = 0; b < a.nbatch; ++b) {
        const int s = b & 1;
        const bool got = dev::mbar_wait_bounded(&bars[s], (b >> 1) & 1);
        if (__syncthreads_or(!got)) {
            if (tid == 0) {
                dev::report(a.status, CT_ETIMEOUT);
                // let the other stage's copy (if any) land before leaving
                if (b + 1 < a.nbatch) dev::mbar_wait_bounded(&bars[s ^ 1], ((b + 1) >> 1) & 1);
            }
            return;
        }
        if (warp_active) {
#pragma unroll
            for (int r = 0; r < kRB; ++r) {
                const uint64_t* rowB = sB + (s * kRB + r) * kTWV;
                const uint64_t* rowM = sM + (s * kRB + r) * kMW;
                uint2 bw[kCPT], mw[12];
                {
                    const uint4* pb = reinterpret_cast<const uint4*>(rowB + 4 * lane);
                    const uint4 q0 = pb[0], q1 = pb[1];
                    bw[0] = make_uint2(q0.x, q0.y); bw[1] = make_uint2(q0.z, q0.w);
                    bw[2] = make_uint2(q1.x, q1.y); bw[3] = make_uint2(q1.z, q1.w);
                    const uint4* pm = reinterpret_cast<const uint4*>(rowM + mstart);
#pragma unroll
                    for (int k = 0; k < 6; ++k) {
                        const uint4 q = pm[k];
                        mw[2 * k] = make_uint2(q.x, q.y);
                        mw[2 * k + 1] = make_uint2(q.z, q.w);
                    }
                }
#pragma unroll
                for (int c = 0; c < kCPT; ++c) {
#pragma unroll
                    for (int p = 0; p < 4; ++p) {
                        const int j0 = 2 * p, j1 = 2 * p + 1;
                        const int k0 = DIR == 0 ? c - j0 + 8 : c + j0;
                        const int k1 = DIR == 0 ? c - j1 + 8 : c + j1;
                        const uint32_t e0 = __popc(bw[c].x ^ mw[k0].x) + __popc(bw[c].y ^ mw[k0].y);
                        const uint32_t e1 = __popc(bw[c].x ^ mw[k1].x) + __popc(bw[c].y ^ mw[k1].y);
                        const uint32_t P = e0 | (e1 << 16);
                        V[c][p] = V[c][p] + P - ring[r][c][p];
                        ring[r][c][p] = P;
                    }
                }
                const int i = b * kRB + r;  // cost row index since ye0
                const int oy = i - 2 * kAR;
                if (oy >= 0 && oy < a.th) {
                    uint32_t C[kCPT][4];
#pragma unroll
                    for (int p = 0; p < 4; ++p) {
                        const uint32_t h0 = __shfl_up_sync(0xffffffffu, V[2][p], 1);
                        const uint32_t h1 = __shfl_up_sync(0xffffffffu, V[3][p], 1);
                        const uint32_t h4 = __shfl_down_sync(0xffffffffu, V[0][p], 1);
                        const uint32_t h5 = __shfl_down_sync(0xffffffffu, V[1][p], 1);
                        C[0][p] = h0 + h1 + V[0][p] + V[1][p] + V[2][p];
                        C[1][p] = C[0][p] + V[3][p] - h0;
                        C[2][p] = C[1][p] + h4 - h1;
                        C[3][p] = C[2][p] + h5 - V[0][p];
                    }
#pragma unroll
                    for (int c = 0; c < kCPT; ++c) {
                        const int v = 4 * lane + c;
                        if (v < kAR || v >= kTWV - kAR) continue;
                        uint32_t k[4];
#pragma unroll
                        for (int p = 0; p < 4; ++p) k[p] = (C[c][p] << 5) + dconst[p];
                        if (!interior) {
                            const int x = xs + v;
                            int lim = DIR == 0 ? x - kAR : a.W - 1 - kAR - x;
                            lim = min(lim, a.D - 1);
#pragma unroll
                            for (int p = 0; p < 4; ++p) {
                                const int dlo = dw + 2 * p;
                                k[p] |= (dlo > lim ? 0x0000FFFFu : 0u) | (dlo + 1 > lim ? 0xFFFF0000u : 0u);
                            }
                        }
                        uint32_t m = dev::min3_u16x2(k[0], k[1], k[2]);
                        m = dev::min_u16x2(m, k[3]);
                        const uint32_t k16 = min(m & 0xFFFFu, m >> 16);
                        const uint32_t key = ((k16 & 0xFFE0u) << 11) | ((k16 & 31u) + dgroup);
                        atomicMin(&sKey[oy * kTWO + v - kAR], key);
                    }
                }
            }
        }
        __syncthreads();  // every warp is done with stage s
        if (tid == 0 && b + 2 < a.nbatch) {
            dev::fence_proxy_async();
            dev::mbar_arrive_expect_tx(&bars[s], kBytesB + kBytesM);
            dev::tma_load_2d(sB + s * kRB * kTWV, &tmB, xs, ye0 + (b + 2) * kRB, &bars[s]);
            dev::tma_load_2d(sM + s * kRB * kMW, &tmM, ms, ye0 + (b + 2) * kRB, &bars[s]);
        }
    }

    // Output: direct when this CTA saw every disparity, else global merge.
    const bool direct = gridDim.z == 1;
    for (int idx = tid; idx < a.th * kTWO; idx += kNT) {
        const int oy = idx / kTWO, ox = idx - oy * kTWO;
        const int x = xs + kAR + ox, y = y0 + oy;
        if (x >= a.W || y >= a.H) continue;
        const uint32_t key = sKey[idx];
        if (direct) {
            const bool valid = x >= kAR && x < a.W - kAR && y >= kAR && y < a.H - kAR;
            store_disp(a.out, a.out_pitch, a.out_type, x, y, valid, key);
        } else {
            atomicMin(&a.keys[(size_t)y * a.W + x], key);
        }
    }
}

// Converts merged keys to disparities and resets the keys for the next call.
// (static: each translation unit that launches it has its own copy.)
static __global__ void keys_finalize_kernel(uint32_t* keys, int W, int H, int r, void* out, size_t out_pitch,
                                     int out_type) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    if (x >= W) return;
    uint32_t* kp = &keys[(size_t)y * W + x];
    const uint32_t key = *kp;
    *kp = 0xFFFFFFFFu;
    const bool valid = x >= r && x < W - r && y >= r && y < H - r;
    store_disp(out, out_pitch, out_type, x, y, valid, key);
}

}  // namespace cm
}  // namespace ct
