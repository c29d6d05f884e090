// census_tile.cuh — one 64 x 32 tile of the 9x7 census transform, shared by
// the single-image census kernel and the batched census kernel.
//
// The tile plus its halo (16 bytes left/right for the TMA x alignment, 3 rows
// above and below) arrives in shared memory with one 2D TMA load. Each
// thread walks 8 rows of one column with a sliding 7 x 9 window; every
// descriptor bit is built with a subtract and a funnel shift (the sign of
// centre - neighbour is "neighbour > centre"), positions in raster order to
// bits 62..0, bit 63 = 0 (the 64-bit generalisation of
// CensusTransform.cu:103-119). Pixels closer than 4 columns / 3 rows to the
// border get 0.
#pragma once

#include "ct_device.cuh"
#include "census_match.cuh"

namespace ct {
namespace census {

constexpr int kTX = 64;   // tile columns
constexpr int kTY = 32;   // tile rows
constexpr int kPY = 8;    // rows per thread
constexpr int kNT = kTX * (kTY / kPY);  // 256 threads
constexpr int kBoxW = kTX + 32;         // 16 halo bytes each side (TMA x alignment)
constexpr int kBoxH = kTY + 6;

// Shared memory the tile needs: the staged image box and one mbarrier.
struct TileSmem {
    uint8_t tile[kBoxH * kBoxW];
    uint64_t bar;
};

// Computes the descriptors of the tile at (x0, y0). planar = 1 writes the
// matcher's pair-planar layout (cm::planar_index), else row-major with
// out_pitch elements per row. Returns false if the tile load timed out (the
// status word is set); all threads of the CTA return the same value.
__device__ __forceinline__ bool census_tile(const CUtensorMap* tm_img, int W, int H, int x0, int y0, uint64_t* out,
                                            size_t out_pitch, int planar, int32_t* status, TileSmem& s) {
    const int tid = threadIdx.x;
    if (tid == 0) {
        dev::mbar_init(&s.bar, 1);
        dev::fence_barrier_init();
    }
    __syncthreads();
    if (tid == 0) {
        dev::mbar_arrive_expect_tx(&s.bar, kBoxW * kBoxH);
        dev::tma_load_2d(s.tile, tm_img, x0 - 16, y0 - 3, &s.bar);
    }
    const bool got = dev::mbar_wait_bounded(&s.bar, 0);
    if (__syncthreads_or(!got)) {
        if (tid == 0) dev::report(status, CT_ETIMEOUT);
        return false;
    }
    const int tx = tid % kTX, ty = tid / kTX;
    const int x = x0 + tx;
    if (x >= W) return true;
    // sliding 7 x 9 window (values as int), rows advance one per pixel
    int w[7][9];
    const uint8_t* base = s.tile + (ty * kPY) * kBoxW + (16 + tx - 4);
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int c = 0; c < 9; ++c) w[r + 1][c] = base[r * kBoxW + c];
#pragma unroll
    for (int p = 0; p < kPY; ++p) {
#pragma unroll
        for (int r = 0; r < 6; ++r)
#pragma unroll
            for (int c = 0; c < 9; ++c) w[r][c] = w[r + 1][c];
#pragma unroll
        for (int c = 0; c < 9; ++c) w[6][c] = base[(p + 6) * kBoxW + c];
        const int y = y0 + ty * kPY + p;
        if (y >= H) break;
        const int ctr = w[3][4];
        uint32_t hi = 0, lo = 0;
        int k = 0;
#pragma unroll
        for (int r = 0; r < 7; ++r)
#pragma unroll
            for (int c = 0; c < 9; ++c, ++k) {
                const uint32_t t = uint32_t(ctr - w[r][c]);  // sign bit = neighbour > centre
                if (k < 31) hi = __funnelshift_l(t, hi, 1);
                else lo = __funnelshift_l(t, lo, 1);
            }
        const bool inside = x >= 4 && x < W - 4 && y >= 3 && y < H - 3;
        const uint64_t d = inside ? ((uint64_t(hi) << 32) | lo) : 0ull;
        out[planar ? cm::planar_index(x, y, W) : (size_t)y * out_pitch + x] = d;
    }
    return true;
}

}  // namespace census
}  // namespace ct
