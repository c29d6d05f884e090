// ncc_tc.cuh — the NCC matcher (match_ncc.cu) with its window cross sums on
// the tensor cores. Included by match_ncc.cu after the CUDA-core kernel; the
// scores, ranking and merge are the same, so are the maps.
//
// For output row y, pixel x and match column x' the window cross sum is
//   C(x, x') = sum over rows r = y-R .. y+R of sum over i = -R .. R of
//              L(x + i, r) R(x' + i, r),
// i.e. for one image row r a product of two matrices: A_r (pixels x, one row
// each holding the 2R+1 pixels of its window row) times B_r^T (match columns
// x', the same). A CTA owns 128 output pixels x0 .. x0+127 of a strip of
// rows and 128 disparities, i.e. match columns xb .. xb+255 (xb = x0 - dmin -
// dz0 - 127): one tcgen05.mma of M = 128, N = 256, K = 16 (f16 operands,
// exact for 8-bit pixels; fp32 accumulation, exact for the 11x11 sums of
// products < 2^24) per image row. The accumulator in TMEM keeps the running
// window sum down the strip: D(y+1) = D(y) + A_{y+R+1} B_{y+R+1}^T -
// A_{y-R} B_{y-R}^T, the subtraction by the descriptor's negate-A bit, so a
// row costs two MMAs. Operands are K-major, no swizzle: pixel row i of a
// panel at i * 16 bytes, the second 8-element K chunk one panel column
// (rows x 16 bytes) further. They are built in shared memory from two staged
// image rows per step (bytes -> f16 through the exponent of 1024); the
// strip's first window is built at once and summed by one chain of 2R+1
// MMAs.
//
// Epilogue: TMEM lane m = pixel x0 + m holds C(x, x') for all 256 columns;
// its disparities d = m + 127 - n (column n) form a 128-wide band. 16 warps:
// lane quarter q = warp % 4 (the lanes a warp may read), column slice h =
// warp / 4 of the quarter's band (40 columns each: 32 q + 40 h ..), read with
// one 32-column and one 8-column tcgen05.ld per row. Ranking as the CUDA-core
// kernel, by the estimate num * rsqrt(vy), num = n C - Sx Sy, here in fp32
// with Sx Sy split into its rounded product and that product's exact error
// (an fma), so that the estimate's error is relative only (~1e-6); every
// disparity whose estimate lies within 4e-6 of the thread's best is scored
// exactly (the IEEE score of the CUDA-core kernel, from the exact integer C),
// so the exact argmax over the thread's disparities is always among them.
// The 4 column slices' keys of a pixel merge in shared memory per row; for
// D > 128 the gridDim.z CTAs' keys merge by atomicMax in global memory with
// the last-arriver merge of the CUDA-core kernel. After each row's barrier
// warp 0 issues the window update, slices 1 and 2 build the operand panels
// of the update after next, slice 3 the column records, slice 0 writes the
// outputs and the pixel records.
#pragma once

#include <type_traits>

namespace ct {
namespace ncc {
namespace tc {

constexpr int kM = 128;    // output pixels per tile = MMA M = TMEM lanes
constexpr int kN = 256;    // match columns per tile = MMA N = accumulator columns
constexpr int kDB = 128;   // disparities per CTA
constexpr int kNT = 512;   // 16 warps: 4 per TMEM lane quarter
constexpr int kCols = 40;  // accumulator columns a thread ranks per row
constexpr int kPA = kM * 16 * 2, kPB = kN * 16 * 2;  // panel bytes (K = 16 f16)
constexpr int kPanel = kPA + kPB;                    // one image row's A and B panels
constexpr int kSet = 2 * kPanel;                     // entering + leaving row
// staged bytes of one image row, as aligned words: the left view from x0 - 8
// (x0 - R .. x0 + 127 + R at byte 8 - R), the right view from xb - R rounded
// down to 4 bytes (xb - R .. xb + 255 + R at byte (xb - R) & 3)
constexpr int kSL = kM + 24, kSR = kN + 20;
static_assert(kSL % 4 == 0 && kSR % 4 == 0 && kSL >= kM + 8 + 2 * 7 && kSR >= kN + 3 + 2 * 7, "staged words");
constexpr int kStage = 2 * (kSL + kSR);              // entering + leaving row
// shared memory
constexpr int kOffSet = 0;                        // 2 panel sets
constexpr int kOffStage = 2 * kSet;               // 2 staging buffers
constexpr int kOffCol = kOffStage + 2 * kStage;   // 3 rows x kN column records (int4)
constexpr int kOffSy = kOffCol + 3 * kN * 16;     // 3 rows x kN column sums Sy
constexpr int kOffPix = kOffSy + 3 * kN * 4;      // 3 rows x kM pixel records (int4)
constexpr int kOffKey = kOffPix + 3 * kM * 16;    // 2 rows x 4 column slices x kM keys
constexpr int kOffBar = kOffKey + 2 * 4 * kM * 8; // MMA completion
constexpr int kOffSlot = kOffBar + 8;             // TMEM address, group-last flag
// the strip's first window: its 2R+1 rows' panels and staged bytes
constexpr int kOffInit = (kOffSlot + 16 + 1023) / 1024 * 1024;
template <int R>
constexpr int smem_bytes() { return kOffInit + (2 * R + 1) * (kPanel + kSL + kSR); }
static_assert(kOffStage % 1024 == 0 && kOffCol % 16 == 0 && kOffPix % 16 == 0 && kOffKey % 8 == 0 &&
                  kOffBar % 8 == 0, "alignment");
constexpr uint32_t kTmemCols = 256;

// Instruction descriptor, kind::f16: D fp32 (bit 4), A and B f16 (bits 7, 10
// = 0), negate A (bit 13), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t idesc(bool negate_a) {
    return (1u << 4) | (uint32_t(negate_a) << 13) | (uint32_t(kN >> 3) << 17) | (uint32_t(kM >> 4) << 24);
}
// Shared-memory matrix descriptor: start, leading byte offset (the next K
// chunk), stride byte offset 128 (the next 8 rows), version 1, no swizzle.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo) {
    return uint64_t((saddr >> 4) & 0x3FFF) | (uint64_t((lbo >> 4) & 0x3FFF) << 16) | (uint64_t(128 >> 4) << 32) |
           (uint64_t(1) << 46);
}
// D += A B^T (accumulate) or D = A B^T, issued by one elected lane of a
// converged warp.
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t id, bool acc) {
    asm volatile(
        "{\n.reg .pred p, e;\nsetp.ne.b32 p, %4, 0;\nelect.sync _|e, 0xffffffff;\n"
        "@e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(id), "r"(uint32_t(acc))
        : "memory");
}
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile(
        "{\n.reg .pred e;\nelect.sync _|e, 0xffffffff;\n"
        "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n}\n" ::"r"(
            dev::smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Columns taddr .. taddr + 39 of this thread's lane, waited for.
__device__ __forceinline__ void ld40(uint32_t taddr, float (&v)[kCols]) {
    uint32_t r[kCols];
    asm volatile(
        "{\n"
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,"
        "%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%40];\n"
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%32,%33,%34,%35,%36,%37,%38,%39}, [%41];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        "}\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39])
        : "r"(taddr), "r"(taddr + 32)
        : "memory");
#pragma unroll
    for (int k = 0; k < kCols; ++k) v[k] = __uint_as_float(r[k]);
}

// Column taddr of this thread's lane, waited for.
__device__ __forceinline__ float ld1(uint32_t taddr) {
    uint32_t r;
    asm volatile(
        "{\n"
        "tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        "}\n"
        : "=r"(r)
        : "r"(taddr)
        : "memory");
    return __uint_as_float(r);
}

// Two staged bytes -> an f16x2 of their values (exact: 1024 + b - 1024).
__device__ __forceinline__ uint32_t bytes_f16x2(uint32_t lo, uint32_t hi) {
    const uint32_t h = (lo | (hi << 16)) | 0x64006400u;
    uint32_t d;
    asm("sub.rn.f16x2 %0, %1, %2;" : "=r"(d) : "r"(h), "r"(0x64006400u));
    return d;
}

// One pixel row of a panel: the 2R+1 staged bytes src[0 ..] as f16, then
// zeros up to K = 16; chunk 0 at dst, chunk 1 at dst + lbo.
template <int R>
__device__ __forceinline__ void build_row(const uint8_t* src, unsigned char* dst, int lbo) {
    constexpr int K = 2 * R + 1;
    uint32_t w[8];
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const uint32_t lo = 2 * p < K ? src[2 * p] : 0u;
        const uint32_t hi = 2 * p + 1 < K ? src[2 * p + 1] : 0u;
        w[p] = 2 * p < K ? bytes_f16x2(lo, hi) : 0u;
    }
    *reinterpret_cast<uint4*>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
    *reinterpret_cast<uint4*>(dst + lbo) = make_uint4(w[4], w[5], w[6], w[7]);
}

}  // namespace tc

// One CTA: pixels x0 .. x0+127 (x0 = 128 blockIdx.x), output rows y0 ..
// y0+th-1 (y0 = th blockIdx.y), relative disparities dz0 .. dz0+127 (dz0 =
// 128 blockIdx.z). Same outputs as ncc_match_kernel<R> without a guide.
template <int R>
__global__ void __launch_bounds__(tc::kNT, 1)
    ncc_tc_kernel(const uint8_t* __restrict__ Limg, size_t pl, const uint8_t* __restrict__ Rimg, size_t pr, Args a) {
    using namespace tc;
    constexpr int n = (2 * R + 1) * (2 * R + 1);
    constexpr int kSB = kSL + kSR;  // staged bytes of one image row
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kOffBar);
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + kOffSlot);
    int4* colrec = reinterpret_cast<int4*>(smem + kOffCol);
    int* colsy = reinterpret_cast<int*>(smem + kOffSy);
    unsigned long long* skey = reinterpret_cast<unsigned long long*>(smem + kOffKey);
    int4* pixrec = reinterpret_cast<int4*>(smem + kOffPix);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int q = warp & 3, h = warp >> 2;
    const int m = 32 * q + lane;           // this thread's pixel = TMEM lane
    const int c0 = 32 * q + kCols * h;     // first accumulator column it ranks
    const int x0 = blockIdx.x * kM, x = x0 + m;
    const int y0 = blockIdx.y * a.th;
    const int rows = min(a.th, a.H - y0);
    const int dz0 = blockIdx.z * kDB;
    const int nd = min(kDB, a.D - dz0);
    const int xb = x0 - a.dmin - dz0 - (kDB - 1);  // match column of accumulator column 0

    if (tid == 0) {
        dev::mbar_init(bar, 1);
        dev::fence_barrier_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dev::smem_u32(slot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = slot[0];
    const uint32_t sbase = dev::smem_u32(smem);
    uint32_t phase = 0;   // MMA commits waited for
    uint32_t issued = 0;  // MMA commits issued (counted by every thread)
    bool failed = false;

    // Word wi of a staging buffer: half s = wi / kWB (0 the entering row, 1
    // the leaving row), word w = wi % kWB: the left view from x0 - 8 (w <
    // kSL / 4), else the right view from xr; bytes outside the image read 0.
    // Image pointers and pitches are 16-byte aligned and the starts are
    // multiples of 4, so a word starting inside a row lies inside its pitch.
    constexpr int kWB = kSB / 4;
    const int xr = (xb - R) & ~3, oL = 8 - R, oR = (xb - R) - xr;
    auto fetch_word = [&](int wi, int r_in, int r_out) -> uint32_t {
        const int s = wi >= kWB, w = wi - s * kWB, r = s ? r_out : r_in;
        const bool left = w < kSL / 4;
        const int xx = left ? x0 - 8 + 4 * w : xr + 4 * (w - kSL / 4);
        if (r < 0 || r >= a.H || xx < 0 || xx >= a.W) return 0u;
        uint32_t v = left ? *reinterpret_cast<const uint32_t*>(Limg + (size_t)r * pl + xx)
                          : *reinterpret_cast<const uint32_t*>(Rimg + (size_t)r * pr + xx);
        if (xx + 4 > a.W) v &= 0xFFFFFFFFu >> (8 * (xx + 4 - a.W));  // bytes at x >= W read 0
        return v;
    };
    // the whole staging buffer b (start of the strip)
    auto stage_rows = [&](int b, int r_in, int r_out) {
        uint32_t* st = reinterpret_cast<uint32_t*>(smem + kOffStage + b * kStage);
        for (int i = tid; i < 2 * kWB; i += tc::kNT) st[i] = fetch_word(i, r_in, r_out);
    };
    // panel row k of panel set p (k < 2 (kM + kN): half k / (kM + kN), A rows
    // first) from staging buffer b
    auto build_item = [&](int p, int b, int k) {
        const int s = k >= kM + kN, i = k - s * (kM + kN);
        const uint8_t* src = smem + kOffStage + b * kStage + s * kSB;
        unsigned char* set = smem + kOffSet + p * kSet;
        if (i < kM) tc::build_row<R>(src + oL + i, set + s * kPA + i * 16, kM * 16);
        else tc::build_row<R>(src + kSL + oR + (i - kM), set + 2 * kPA + s * kPB + (i - kM) * 16, kN * 16);
    };
    auto build_all = [&](int p, int b) {
        for (int k = tid; k < 2 * (kM + kN); k += tc::kNT) build_item(p, b, k);
        dev::fence_proxy_async();  // generic-proxy writes -> the tensor core's reads
    };
    auto wait_mma = [&]() {
        const bool ok = dev::mbar_wait_bounded(bar, phase & 1);
        if (ok) ++phase;
        return ok;
    };
    auto desc_a = [&](int p, int s) { return tc::sdesc(sbase + kOffSet + p * kSet + s * kPA, kM * 16); };
    auto desc_b = [&](int p, int s) { return tc::sdesc(sbase + kOffSet + p * kSet + 2 * kPA + s * kPB, kN * 16); };
    // column cx of output row y: its Sy, vy (loaded a step before the record
    // is stored); columns whose window leaves the image are outside every
    // thread's column range below (record 0)
    auto fetch_col = [&](int cx, int y, int& sy, int& vy) {
        const int xx = xb + cx;
        sy = 0;
        vy = -1;  // not a searchable column
        if (xx >= R && xx < a.W - R && y >= 0 && y < a.H) {
            const size_t o = (size_t)y * a.W + xx;
            sy = a.Sy[o];
            vy = a.Vy[o];
        }
    };
    // column record {r, float(Sy), vy, 0} (r ~ 1 / sqrt(vy)) and Sy of
    // column cx in buffer b
    auto store_col = [&](int cx, int b, int sy, int vy) {
        int4 rec = make_int4(0, 0, 0, 0);
        if (vy >= 0)
            rec = make_int4(__float_as_int(vy > 0 ? rsqrtf(__int2float_rn(vy)) : 0.0f),
                            __float_as_int(__int2float_rn(sy)), vy, 0);
        colrec[b * kN + cx] = rec;
        colsy[b * kN + cx] = sy;
    };

    // Duties after the barrier of a step, spread so that every warp's step
    // takes about as long (the warps of column slices 0 and 3 rank with the
    // range test): slices 1, 2 build the panels (3 panel rows a thread),
    // slice 3 the column records (2 columns a thread), slice 0 the outputs,
    // every thread one or two staged bytes.
    const bool builder = h == 1 || h == 2;
    const int bk0 = tid - kM;  // first panel row of a builder: bk0, bk0 + 256, bk0 + 512
    const bool colder = h == 3;
    const int cx0 = tid - 3 * kM;  // columns of slice 3's threads: cx0, cx0 + 128
    auto build_mine = [&](int p, int b) {
        if (!builder) return;
#pragma unroll
        for (int t = 0; t < 3; ++t) build_item(p, b, bk0 + 2 * kM * t);
        dev::fence_proxy_async();
    };

    // ---- the strip's first window D(y0), rows y0 - R .. y0 + R: all rows
    // staged and built at once (panels of their own after the rest of the
    // shared memory), one MMA each, one commit. With it: the rows of the
    // first update (entering y0 + R + 1, leaving y0 - R) into staging buffer
    // 1 and panel set 1, the first two rows' column records.
    {
        constexpr int NW = 2 * R + 1;
        uint8_t* istage = smem + kOffInit + NW * kPanel;
        for (int i = tid; i < NW * kWB; i += tc::kNT) {
            const int k = i / kWB;
            reinterpret_cast<uint32_t*>(istage)[i] = fetch_word(i - k * kWB, y0 - R + k, 0);
        }
        stage_rows(1, y0 + R + 1, y0 - R);
        for (int cx = tid; cx < kN; cx += tc::kNT) {
            int sy, vy;
            fetch_col(cx, y0, sy, vy);
            store_col(cx, 0, sy, vy);
            fetch_col(cx, y0 + 1, sy, vy);
            store_col(cx, 1, sy, vy);
        }
        __syncthreads();
        for (int i = tid; i < NW * (kM + kN); i += tc::kNT) {
            const int k = i / (kM + kN), t = i - k * (kM + kN);
            const uint8_t* src = istage + k * kSB;
            unsigned char* pan = smem + kOffInit + k * kPanel;
            if (t < kM) tc::build_row<R>(src + oL + t, pan + t * 16, kM * 16);
            else tc::build_row<R>(src + kSL + oR + (t - kM), pan + kPA + (t - kM) * 16, kN * 16);
        }
        build_all(1, 1);  // ends with the proxy fence
        tc::fence_before();
        __syncthreads();
        if (warp == 0) {
            tc::fence_after();
#pragma unroll
            for (int k = 0; k < NW; ++k) {
                const uint32_t pa = sbase + uint32_t(kOffInit + k * kPanel);
                tc::mma(tmem, tc::sdesc(pa, kM * 16), tc::sdesc(pa + kPA, kN * 16), tc::idesc(false), k > 0);
            }
            tc::commit(bar);
        }
        ++issued;
        // staging buffer 0: the rows of the update after (y0 + R + 2 in,
        // y0 - R + 1 out)
        stage_rows(0, y0 + R + 2, y0 - R + 1);
    }
    // loads in flight across a step: the staged words of the rows after next
    // (word tid of a buffer) and the column inputs of row y + 2
    static_assert(2 * kWB <= tc::kNT, "one staged word a thread");
    uint32_t pf0 = tid < 2 * kWB ? fetch_word(tid, y0 + R + 3, y0 - R + 2) : 0u;
    int pf_sy0 = 0, pf_vy0 = -1, pf_sy1 = 0, pf_vy1 = -1;
    if (colder) {
        fetch_col(cx0, y0 + 2, pf_sy0, pf_vy0);
        fetch_col(cx0 + kM, y0 + 2, pf_sy1, pf_vy1);
    }

    // Pixel records {Sx, float(vx), threshold Tx, inside} of output row y:
    // slice 0's thread of pixel m loads them a step before it stores them,
    // two steps before they are read.
    auto fetch_pix = [&](int y, int4& p) {
        const bool in = x >= R && x < a.W - R && y >= R && y < a.H - R;
        const size_t o = (size_t)(in ? y : R) * a.W + (in ? x : R);
        p = make_int4(a.Sx[o], __float_as_int(__int2float_rn(a.Vx[o])), a.Tx[o], in);
    };
    int4 pf_pix = make_int4(0, 0, 0, 0);
    if (h == 0) {
        int4 p;
        fetch_pix(y0, p);
        pixrec[m] = p;
        fetch_pix(y0 + 1, p);
        pixrec[kM + m] = p;
        fetch_pix(y0 + 2, pf_pix);
    }
    __syncthreads();
    // this thread's disparities: d = m + 127 - n for its columns n = c0 + j;
    // searched iff jlo <= j <= jhi: d < nd, and the matched window inside the
    // image (R <= xb + n < W - R)
    const int jlo = max(m + kDB - nd - c0, R - xb - c0);
    const int jhi = min(m + kDB - 1 - c0, a.W - R - 1 - xb - c0);

    // Step oy (output row y = y0 + oy): rank row y from D(y), then one
    // barrier, then the update D(y) -> D(y + 1), the outputs of row y and the
    // operands of the steps ahead. The rare near-tie path re-reads the
    // accumulator, which stays D(y) until that barrier.
    for (int oy = 0; oy < rows && !failed; ++oy) {
        const int y = y0 + oy;
        const int4 pr = pixrec[(oy % 3) * kM + m];
        const int sx = pr.x, tx = pr.z;
        const float fvx = __int_as_float(pr.y);
        const bool pok = pr.w != 0;
        const uint32_t tlane = tmem + (uint32_t(32 * q) << 16);
        // ---- the window sums of row y
        const bool ok = phase < issued ? wait_mma() : true;
        tc::fence_after();
        const int4* cr = colrec + (oy % 3) * kN + c0;
        const int* csy = colsy + (oy % 3) * kN + c0;
        const float sxf = __int2float_rn(sx);
        // Estimate of column j from its sum c: num * r with num = n c - Sx Sy
        // in fp32 with Sx Sy split exactly into a rounded product and its
        // error (an fma), so that the estimate's error is relative only (at
        // most 2^-23 of num, 2^-24 of the product and the error of r, ~1e-6
        // in all); 0 when the score is +0 by sigma_x sigma_y < 1, -inf
        // outside the thread's range (MASK).
        auto est_of = [&](float c, int j, const int4& rec, bool mask) {
            const float syf = __int_as_float(rec.y);
            const float ph = __fmul_rn(sxf, syf);
            const float plo = fmaf(sxf, syf, -ph);
            const float num = __fsub_rn(fmaf(float(n), c, -ph), plo);
            const float e = rec.z >= tx ? num * __int_as_float(rec.x) : 0.0f;
            return (!mask || (pok && j >= jlo && j <= jhi)) ? e : -INFINITY;
        };
        // best estimate (ties: the lowest d, i.e. the highest j) and the
        // second largest, in 4 independent chains
        float best, cbest, v2;
        int jbest;
        {
            float C[kCols];
            tc::ld40(tlane + uint32_t(c0), C);  // garbage if the wait gave up (then unused)
            float bv[4], bc[4], t2[4];
            int bj[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                bv[k] = t2[k] = -INFINITY;
                bc[k] = 0.0f;
                bj[k] = 0;
            }
            // every lane's columns all searched: no range test
            const bool full = __all_sync(0xffffffffu, pok && jlo <= 0 && jhi >= kCols - 1);
            auto pass = [&](auto masked) {
#pragma unroll
                for (int j = 0; j < kCols; ++j) {
                    const int k = j & 3;
                    const float v = est_of(C[j], j, cr[j], decltype(masked)::value);
                    t2[k] = fmaxf(t2[k], fminf(bv[k], v));
                    const bool up = v >= bv[k];
                    bv[k] = up ? v : bv[k];
                    bc[k] = up ? C[j] : bc[k];
                    bj[k] = up ? j : bj[k];
                }
            };
            if (full) pass(std::integral_constant<bool, false>{});
            else pass(std::integral_constant<bool, true>{});
            best = bv[0];
            cbest = bc[0];
            jbest = bj[0];
#pragma unroll
            for (int k = 1; k < 4; ++k) {
                const bool take = bv[k] > best || (bv[k] == best && bj[k] > jbest);
                best = take ? bv[k] : best;
                cbest = take ? bc[k] : cbest;
                jbest = take ? bj[k] : jbest;
            }
            const float a0 = fmaxf(bv[0], bv[1]), b0 = fminf(bv[0], bv[1]);
            const float a1 = fmaxf(bv[2], bv[3]), b1 = fminf(bv[2], bv[3]);
            v2 = fmaxf(fmaxf(fminf(a0, a1), fmaxf(b0, b1)), fmaxf(fmaxf(t2[0], t2[1]), fmaxf(t2[2], t2[3])));
        }
        // Another column j can hold the exact maximum (the IEEE scores round
        // the same quantity num / sqrt(vx vy), within a few 2^-24) only if
        // its estimate is above best - 4e-6 |best|; exact estimates (0, the
        // score +0) are equal only to each other, and those went to the
        // lowest d above. Such a j exists iff the second largest estimate is
        // above that bound.
        const float lower = best - 4e-6f * fabsf(best);
        const bool searched = best > -INFINITY;
        const bool others = ok && searched && v2 > lower;
        auto d_of = [&](int j) { return m + kDB - 1 - (c0 + j) + dz0; };  // relative to dmin
        // IEEE score of column j with window sum c (an exact integer in fp32)
        auto exact_key = [&](float c, int j) {
            const int vy = cr[j].z;
            float sc = 0.0f;  // +0 when sigma_x sigma_y < 1
            if (vy >= tx) {
                const int num = n * __float2int_rn(c) - sx * csy[j];
                sc = __fdiv_rn(__int2float_rn(num), __fsqrt_rn(__fmul_rn(fvx, __int2float_rn(vy))));
            }
            return ((unsigned long long)ordered(sc) << 32) | (0xFFFFFFFFu - uint32_t(d_of(j)));
        };
        unsigned long long key = searched ? exact_key(cbest, jbest) : 0ull;
        // those columns (rare: a few warps in a thousand): the warp re-reads
        // every column (a warp-wide TMEM load) and scores the candidates
        if (__any_sync(0xffffffffu, others)) {
#pragma unroll 1
            for (int j = 0; j < kCols; ++j) {
                const float c = tc::ld1(tlane + uint32_t(c0 + j));
                if (others && j != jbest && est_of(c, j, cr[j], true) > lower) {
                    const unsigned long long k2 = exact_key(c, j);
                    key = k2 > key ? k2 : key;
                }
            }
        }
        skey[((oy & 1) * 4 + h) * kM + m] = key;  // this column slice's best for pixel m
        tc::fence_before();
        // the accumulator is read, the keys of row y are in, the operands of
        // this step's update are in place
        if (__syncthreads_or(!ok)) { failed = true; break; }
        // ---- D(y + 1) = D(y) + entering row - leaving row
        const int pb = (oy + 1) & 1;  // panel set of that update
        if (oy + 1 < rows) {
            if (warp == 0) {
                tc::fence_after();
                tc::mma(tmem, desc_a(pb, 0), desc_b(pb, 0), tc::idesc(false), true);
                tc::mma(tmem, desc_a(pb, 1), desc_b(pb, 1), tc::idesc(true), true);
                tc::commit(bar);
            }
            ++issued;
        }
        // ---- outputs of row y (slice 0: its own pixel)
        if (h == 0) {
            const unsigned long long* kp = &skey[(oy & 1) * 4 * kM + m];
            const unsigned long long kk = max(max(kp[0], kp[kM]), max(kp[2 * kM], kp[3 * kM]));
            if (x < a.W) {
                if (gridDim.z == 1) store_ncc(a, x, y, x >= R && x < a.W - R && y >= R && y < a.H - R, kk);
                else if (kk) atomicMax(&a.keys[(size_t)y * a.W + x], kk);
            }
        }
        // ---- operands of the steps ahead: panels of the update after next
        // (set oy & 1, free: D(y) is done) from staging buffer oy & 1, column
        // records of row y + 2 (read after the next barrier), staged rows of
        // the update after that into staging buffer (oy + 1) & 1 (read by the
        // previous step's build)
        if (oy + 2 < rows) build_mine(oy & 1, oy & 1);
        if (oy + 2 < rows && colder) {
            store_col(cx0, (oy + 2) % 3, pf_sy0, pf_vy0);
            store_col(cx0 + kM, (oy + 2) % 3, pf_sy1, pf_vy1);
            fetch_col(cx0, y + 3, pf_sy0, pf_vy0);
            fetch_col(cx0 + kM, y + 3, pf_sy1, pf_vy1);
        }
        if (oy + 3 < rows) {
            if (tid < 2 * kWB) {
                reinterpret_cast<uint32_t*>(smem + kOffStage + ((oy + 1) & 1) * kStage)[tid] = pf0;
                pf0 = fetch_word(tid, y + R + 4, y - R + 3);
            }
        }
        if (oy + 2 < rows && h == 0) {
            pixrec[((oy + 2) % 3) * kM + m] = pf_pix;
            fetch_pix(y + 3, pf_pix);
        }
    }
    if (failed && tid == 0) dev::report(a.status, CT_ETIMEOUT);
    // outstanding MMAs (a failed wait) complete before the TMEM is released
    if (failed && warp == 0)
        for (uint32_t k = phase; k < issued; ++k) dev::mbar_wait_bounded(bar, k & 1);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    if (gridDim.z == 1) return;
    // ---- D split over gridDim.z CTAs: the last of the (strip, column tile)
    // group writes the merged keys as outputs and resets keys and counter
    __threadfence();
    __syncthreads();
    int* last = reinterpret_cast<int*>(slot + 1);
    if (tid == 0) {
        uint32_t* ctr = &a.counters[blockIdx.y * gridDim.x + blockIdx.x];
        const bool l = atomicAdd(ctr, 1u) == gridDim.z - 1;
        if (l) *ctr = 0u;
        *last = l;
    }
    __syncthreads();
    if (!*last) return;
    __threadfence();
    for (int idx = tid; idx < rows * kM; idx += tc::kNT) {
        const int oy = idx / kM, xx = x0 + idx % kM, yy = y0 + oy;
        if (xx >= a.W) continue;
        unsigned long long* kp = &a.keys[(size_t)yy * a.W + xx];
        const unsigned long long key = __ldcg(kp);
        *kp = 0ull;
        store_ncc(a, xx, yy, xx >= R && xx < a.W - R && yy >= R && yy < a.H - R, key);
    }
}

}  // namespace ncc
}  // namespace ct
