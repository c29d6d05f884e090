// guide.cuh — search ranges of the guided (coarse-to-fine) matchers
// (MatcherUseDisparity, BlockMatcherNCC.cu:894-1255, BlockMatcherAW1.cu:996-1180).
//
// Pixels are grouped in 16 x 16 blocks aligned to multiples of 16; pixel
// (x, y) takes the coarse disparity at (x / s, y / s) scaled by s, and a block
// searches only [max(0, min - 4), max + 4] of its pixels' scaled coarse
// disparities, nothing when none of them has one. One thread per block; the
// range is packed lo | hi << 16 (lo > hi: no search), relative to the
// matcher's minimum disparity dmin (clipped at 0).
#pragma once

#include <cstdint>

#include "../../include/ctstereo.h"

namespace ct {
namespace guide {

constexpr int kBlock = 16, kMargin = 4;

template <int kUnused = 0>
__global__ void range_kernel(const void* coarse, size_t pitch, int type, int s, int W, int H, uint32_t* ranges, int gw,
                             int gh, int dmin) {
    const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y;
    if (gx >= gw || gy >= gh) return;
    const int x0 = gx * kBlock, x1 = min(x0 + kBlock, W) - 1;
    const int y0 = gy * kBlock, y1 = min(y0 + kBlock, H) - 1;
    int lo = 1 << 20, hi = -1;
    for (int cy = y0 / s; cy <= y1 / s; ++cy) {
        const char* row = static_cast<const char*>(coarse) + (size_t)cy * pitch;
        for (int cx = x0 / s; cx <= x1 / s; ++cx) {
            int d;
            if (type == CT_PIX_U8) {
                const int v = reinterpret_cast<const uint8_t*>(row)[cx];
                d = v == 0xFF ? -1 : v;
            } else {
                const int v = reinterpret_cast<const uint16_t*>(row)[cx];
                d = (v >= CT_DISP_FIRST && v <= CT_DISP_LAST) ? v - 1 : -1;
            }
            if (d >= 0) {
                lo = min(lo, d * s);
                hi = max(hi, d * s);
            }
        }
    }
    const int rlo = max(0, max(0, lo - kMargin) - dmin), rhi = hi + kMargin - dmin;
    ranges[(size_t)gy * gw + gx] =
        (hi < 0 || rhi < rlo) ? 0x0000FFFFu : (uint32_t(rlo) | (uint32_t(min(rhi, 0xFFFF)) << 16));
}

// Union of the ranges of the blocks that output columns [c0, c1] and rows
// [r0, r1] fall in, reduced over the CTA into uni[0] (lo) / uni[1] (hi):
// every thread of the CTA calls it; returns (lo, hi) with lo > hi when empty.
__device__ __forceinline__ int2 tile_union(const uint32_t* ranges, int gw, int c0, int c1, int r0, int r1, int* uni) {
    if (threadIdx.x == 0) {
        uni[0] = 1 << 20;
        uni[1] = -1;
    }
    __syncthreads();
    const int gx0 = c0 / kBlock, gx1 = c1 / kBlock, gy0 = r0 / kBlock, gy1 = r1 / kBlock;
    const int ngx = gx1 - gx0 + 1;
    for (int i = threadIdx.x; i < ngx * (gy1 - gy0 + 1); i += blockDim.x) {
        const uint32_t g = ranges[(size_t)(gy0 + i / ngx) * gw + gx0 + i % ngx];
        if ((g & 0xFFFFu) <= (g >> 16)) {
            atomicMin(&uni[0], int(g & 0xFFFFu));
            atomicMax(&uni[1], int(g >> 16));
        }
    }
    __syncthreads();
    return make_int2(uni[0], uni[1]);
}

}  // namespace guide
}  // namespace ct
