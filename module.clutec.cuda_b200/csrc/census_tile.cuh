// census_tile.cuh — one 128 x 32 tile of the 9x7 census transform, shared by
// the single-image census kernel and the batched census kernel.
//
// The tile plus its halo (16 bytes left/right for the TMA x alignment, 3 rows
// above and below) arrives in shared memory with one 2D TMA load. Each thread
// computes 4 adjacent pixels x .. x + 3 of 4 rows, 4 pixels per instruction:
// for a window position (dy, dx) the 4 neighbours form one 32-bit word, and
// __vcmpgtu4 against the 4 centres gives one 0x00 / 0xFF byte per pixel
// ("neighbour > centre"). Position k (raster order) is descriptor bit
// 62 - k (bit 63 = 0, the 64-bit generalisation of CensusTransform.cu:103-119);
// a LOP3 moves the compare bytes' bit (62 - k) % 8 into bit-plane word
// acc[(62 - k) / 8], whose byte p then holds descriptor byte (62 - k) / 8 of
// pixel p; a 4 x 4 byte transpose turns the 8 plane words into the 4
// descriptors. Pixels closer than 4 columns / 3 rows to the border get 0.
#pragma once

#include "ct_device.cuh"
#include "census_match.cuh"

namespace ct {
namespace census {

constexpr int kTX = 128;  // tile columns
constexpr int kTY = 32;   // tile rows
constexpr int kPX = 4;    // columns per thread (one 32-bit word)
constexpr int kPY = 4;    // rows per thread
constexpr int kNT = (kTX / kPX) * (kTY / kPY);  // 256 threads: a warp = one row group
constexpr int kBoxW = kTX + 32;         // 16 halo bytes each side (TMA x alignment)
constexpr int kBoxH = kTY + 6;

// Shared memory the tile needs: the staged image box and one mbarrier.
struct TileSmem {
    uint8_t tile[kBoxH * kBoxW];
    uint64_t bar;
};

// 4 x 4 byte transpose: out[p] byte i = in[i] byte p.
__device__ __forceinline__ void transpose4(const uint32_t (&in)[4], uint32_t (&out)[4]) {
    const uint32_t t01l = __byte_perm(in[0], in[1], 0x5140), t01h = __byte_perm(in[0], in[1], 0x7362);
    const uint32_t t23l = __byte_perm(in[2], in[3], 0x5140), t23h = __byte_perm(in[2], in[3], 0x7362);
    out[0] = __byte_perm(t01l, t23l, 0x5410);
    out[1] = __byte_perm(t01l, t23l, 0x7632);
    out[2] = __byte_perm(t01h, t23h, 0x5410);
    out[3] = __byte_perm(t01h, t23h, 0x7632);
}

// Computes the descriptors of the tile at (x0, y0). planar = 1 writes the
// matcher's pair-planar layout (cm::planar_index), else row-major with
// out_pitch elements per row (16-byte aligned rows). Returns false if the
// tile load timed out (the status word is set); all threads of the CTA return
// the same value.
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
    const int gx = tid % (kTX / kPX), gy = tid / (kTX / kPX);
    const int x = x0 + kPX * gx;  // first of this thread's 4 columns
    if (x >= W) return true;
    // per staged row: the words holding columns x - 4 .. x + 7
    const uint32_t* rows = reinterpret_cast<const uint32_t*>(s.tile) + (gy * kPY) * (kBoxW / 4) + 3 + gx;
    uint32_t win[7][3];
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int k = 0; k < 3; ++k) win[r + 1][k] = rows[r * (kBoxW / 4) + k];
#pragma unroll
    for (int p = 0; p < kPY; ++p) {
#pragma unroll
        for (int r = 0; r < 6; ++r)
#pragma unroll
            for (int k = 0; k < 3; ++k) win[r][k] = win[r + 1][k];
#pragma unroll
        for (int k = 0; k < 3; ++k) win[6][k] = rows[(p + 6) * (kBoxW / 4) + k];
        const int y = y0 + gy * kPY + p;
        if (y >= H) break;
        const uint32_t ctr = win[3][1];
        uint32_t acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int r = 0; r < 7; ++r)
#pragma unroll
            for (int c = 0; c < 9; ++c) {
                // neighbours of the 4 pixels at dx = c - 4: bytes c .. c + 3 of words 0 .. 2
                const uint32_t nb = c == 0 ? win[r][0]
                                  : c < 4  ? __byte_perm(win[r][0], win[r][1], 0x3210 + 0x1111 * c)
                                  : c == 4 ? win[r][1]
                                  : c < 8  ? __byte_perm(win[r][1], win[r][2], 0x3210 + 0x1111 * (c - 4))
                                           : win[r][2];
                const uint32_t gt = __vcmpgtu4(nb, ctr);
                const int bit = 62 - (r * 9 + c);
                acc[bit >> 3] |= gt & (0x01010101u << (bit & 7));
            }
        uint32_t lo[4], hi[4];
        transpose4({acc[0], acc[1], acc[2], acc[3]}, lo);
        transpose4({acc[4], acc[5], acc[6], acc[7]}, hi);
        const bool row_in = y >= 3 && y < H - 3;
        uint64_t d[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int xq = x + q;
            d[q] = (row_in && xq >= 4 && xq < W - 4) ? ((uint64_t(hi[q]) << 32) | lo[q]) : 0ull;
        }
        if (x + 3 < W) {  // two 16-byte stores: pixels (x, x+1) and (x+2, x+3)
            uint64_t* p01 = out + (planar ? cm::planar_index(x, y, W) : (size_t)y * out_pitch + x);
            uint64_t* p23 = out + (planar ? cm::planar_index(x + 2, y, W) : (size_t)y * out_pitch + x + 2);
            *reinterpret_cast<ulonglong2*>(p01) = make_ulonglong2(d[0], d[1]);
            *reinterpret_cast<ulonglong2*>(p23) = make_ulonglong2(d[2], d[3]);
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (x + q < W) out[planar ? cm::planar_index(x + q, y, W) : (size_t)y * out_pitch + x + q] = d[q];
        }
    }
    return true;
}

}  // namespace census
}  // namespace ct
