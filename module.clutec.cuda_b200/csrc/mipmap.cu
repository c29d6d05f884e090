// mipmap.cu — disparity mip-maps (CreateDispMipMaps::CDriver,
// CreateDispMipMaps.h:44-80 / CreateDispMipMaps.cu:66-330) in the packed
// mip-map image of _CDeviceSurfMipMap (DeviceSurfMipMap.h:40-150,
// DeviceSurfMipMap.cpp:68-146).
//
// Packed layout (F32, one image): level 0 (W x H) at (0, 0); level k >= 1 at
// (X1, H_1 + ... + H_{k-1}) with X1 = W rounded up to a multiple of 4, so
// every level starts 16-byte aligned; W_{k+1} = (W_k - 1) / 2, H_{k+1} =
// (H_k - 1) / 2; image width X1 + (W - 1) / 2, height H. The maximal level count is
// the number of levels k >= 1 with W_k, H_k > 0 (the reference's count).
//
// Level 0 holds the disparity codes as floats: code c in First .. Last (1 ..
// 0xFFEF) -> float(c), every other code -> 0 (Unknown). Level k + 1 at (x, y):
// the horizontal pass h(x, r) = weighted mean of level k at (2x, r), (2x + 1,
// r), (2x + 2, r) with weights 1, 2, 1 over the entries that are not 0
// (0 if all are), then 0.5 x the same weighted mean of h(x, 2y), h(x, 2y + 1),
// h(x, 2y + 2) (SmoothHorizontalLum / SmoothVerticalLum,
// CreateDispMipMaps.cu:116-238). The sums are formed in the reference's order
// and divided with IEEE division, so the result is bit-identical to it; the
// horizontal pass goes through shared memory instead of a temporary image;
// the division is division-free but rounds identically (div_count).
//
// Launches: the levels are produced two at a time by a tiled kernel: a CTA
// stages a 131 x 35 region of the source level in shared memory (for the
// first launch the code map, converting it and storing level 0 from the
// staged tile), computes its 65 x 17 pixels of the next level there and
// its 32 x 8 pixels of the level after; once the source level fits in
// shared memory (kTailA pixels), one single-CTA launch computes every
// remaining level from shared memory. At 1920x1080 that is three launches
// (levels 0-2, 3-4, 5-8), chained with programmatic stream serialisation.
// HBM-bound: 2 B read + 4 B written per level-0 pixel, 4 B per pixel of the
// smaller levels.
#include "ct_internal.h"

namespace ct {
namespace mip {

constexpr int kTX = 128, kTY = 32;             // source pixels a CTA owns
constexpr int kSX = kTX + 3, kSY = kTY + 3;    // source region a CTA reads (131 x 35)
constexpr int kSXA = kTX + 17;                 // staged row stride (16-byte chunks cover up to 144 columns)
constexpr int kS1X = kTX / 2 + 1, kS1Y = kTY / 2 + 1;  // next level, owned + 1 (65 x 17)
constexpr int kNT = 256;
constexpr int kTailA = 9600;                   // tail: source level at most this many pixels
constexpr int kTailB = kTailA / 4;             // its next level
constexpr int kTailChunks = 4096;              // and at most this many 16-byte chunks (ceil(w / 4) x h)
constexpr int kTailThreads = 1024;

__host__ __device__ inline int next_size(int n) { return (n - 1) / 2; }

__device__ __forceinline__ float code_value(uint32_t c) {
    return (c >= CT_DISP_FIRST && c <= CT_DISP_LAST) ? float(c) : 0.f;
}

// Source element k of a 16-byte chunk as a level value: U8 d -> code d + 1
// (255 -> CannotEvaluate -> 0), U16 codes via code_value, F32 levels as
// stored.
template <typename T>
__device__ __forceinline__ float chunk_value(const uint4& q, int k) {
    const uint32_t word = (&q.x)[k * sizeof(T) / 4];
    if constexpr (sizeof(T) == 1) {
        const uint32_t v = (word >> (8 * (k & 3))) & 0xFFu;
        return v == 0xFFu ? 0.f : float(v + 1u);
    } else if constexpr (sizeof(T) == 2) {
        return code_value((word >> (16 * (k & 1))) & 0xFFFFu);
    } else {
        return __uint_as_float(word);
    }
}

// Stages rows [y0, y0 + rows) x columns [x0, x0 + cols) of a source image
// (16-byte aligned rows; x0 a multiple of 16 / sizeof(T)) into dst (row
// stride dstride floats) as level values, 0 outside sw x sh. Each thread
// issues all its 16-byte loads before converting and storing, so they are in
// flight together. A chunk that starts inside a row ends inside its pitch
// (pitches are multiples of 16 bytes and at least a row), its elements past
// sw are replaced by 0.
template <typename T, int NT, int MAXCHUNKS>
__device__ __forceinline__ void stage(float* dst, int dstride, const char* src, size_t pitch, int sw, int sh,
                                      int x0, int y0, int cols, int rows) {
    constexpr int E = 16 / sizeof(T);
    const int cpr = (cols + E - 1) / E, n = cpr * rows;
    constexpr int kPer = (MAXCHUNKS + NT - 1) / NT;
    uint4 q[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const int i = threadIdx.x + j * NT, r = i / cpr, c = (i - r * cpr) * E, x = x0 + c, y = y0 + r;
        q[j] = (i < n && x < sw && y < sh)
                   ? *reinterpret_cast<const uint4*>(src + (size_t)y * pitch + (size_t)x * sizeof(T))
                   : make_uint4(0, 0, 0, 0);
    }
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const int i = threadIdx.x + j * NT, r = i / cpr, c = (i - r * cpr) * E, x = x0 + c;
        if (i >= n) continue;
#pragma unroll
        for (int k = 0; k < E; ++k)
            if (c + k < cols) dst[r * dstride + c + k] = x + k < sw ? chunk_value<T>(q[j], k) : 0.f;
    }
}

// s / c for a weight count c in {1, 2, 3, 4}, rounded to nearest as the
// reference's IEEE division: 1, 2 and 4 are exact scalings; for 3 the
// quotient is formed in double (relative error below 2^-51) and rounded to
// float once. For a float s = M 2^E (M < 2^24) that is not a multiple of 3,
// s / 3 lies at least 1/6 ulp away from every midpoint between floats (in
// units of half an ulp it is N / 3 against an odd integer, N an integer), so
// that single rounding returns the correctly rounded quotient.
__device__ __forceinline__ float div_count(float s, float c) {
    if (c == 3.f) return __double2float_rn(double(s) * (1.0 / 3.0));
    return __fmul_rn(s, c == 4.f ? 0.25f : c == 2.f ? 0.5f : 1.f);
}

// Weighted 1-2-1 mean of the non-zero entries, in the reference's order.
__device__ __forceinline__ float mean121(float a, float b, float c) {
    float cnt = 0.f, sum = 0.f;
    if (a != 0.f) {
        cnt += 1.f;
        sum += a;
    }
    if (b != 0.f) {
        cnt += 2.f;
        sum = __fadd_rn(sum, __fmul_rn(b, 2.f));
    }
    if (c != 0.f) {
        cnt += 1.f;
        sum += c;
    }
    return cnt > 0.f ? div_count(sum, cnt) : 0.f;
}

// Next-level value from the 3 x 3 block at p (row stride `stride`).
__device__ __forceinline__ float reduce3x3(const float* p, int stride) {
    const float h0 = mean121(p[0], p[1], p[2]);
    const float h1 = mean121(p[stride], p[stride + 1], p[stride + 2]);
    const float h2 = mean121(p[2 * stride], p[2 * stride + 1], p[2 * stride + 2]);
    return __fmul_rn(0.5f, mean121(h0, h1, h2));
}

struct Level {
    float* ptr;  // first pixel of the level in the packed image; w = 0: not written
    int w, h;
};

__device__ __forceinline__ float* row_of(const Level& l, size_t pitch, int y) {
    return reinterpret_cast<float*>(reinterpret_cast<char*>(l.ptr) + (size_t)y * pitch);
}

struct FusedArgs {
    const void* src;   // source level: the code map (T = uint8_t / uint16_t) or a float level
    size_t src_pitch;
    int sw, sh;
    Level l0;          // code source only: level 0 (the converted codes)
    Level l1, l2;      // the two levels below the source
    size_t pitch;      // the packed image's row pitch
};

// CTA (bx, by) owns source pixels [128 bx, 128 bx + 128) x [32 by, 32 by + 32),
// next-level pixels [64 bx, + 64) x [16 by, + 16) and [32 bx, + 32) x
// [8 by, + 8) of the level after (clipped to each level's size; the grid is
// ceil(sw / 128) x ceil(sh / 32), so the owned ranges cover every level).
// A valid pixel of a level only reads valid pixels of the level above, so
// the zero fill outside the source never reaches an output.
template <typename T>
__global__ void __launch_bounds__(kNT) fused_kernel(FusedArgs a) {
    __shared__ float s0[kSY * kSXA];         // source region
    __shared__ float h1[kSY * kS1X];         // its horizontal means (SmoothHorizontalLum)
    __shared__ float s1[kS1Y * kS1X];        // next level
    __shared__ float h2[kS1Y * (kTX / 4)];   // its horizontal means
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
    {
        constexpr int E = 16 / sizeof(T);
        constexpr int kChunks = (kSX + E - 1) / E * kSY;
        stage<T, kNT, kChunks>(s0, kSXA, static_cast<const char*>(a.src), a.src_pitch, a.sw, a.sh, x0, y0, kSX,
                               kSY);
    }
    __syncthreads();
    if constexpr (sizeof(T) < 4) {  // level 0: the owned tile, 4 columns per store
        for (int i = tid; i < kTY * (kTX / 4); i += kNT) {
            const int r = i / (kTX / 4), c = 4 * (i % (kTX / 4)), x = x0 + c, y = y0 + r;
            if (y >= a.sh || x >= a.sw) continue;
            const float* v = &s0[r * kSXA + c];
            float* dst = row_of(a.l0, a.pitch, y) + x;
            if (x + 3 < a.sw) {
                *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
            } else {
                for (int q = 0; q < 4 && x + q < a.sw; ++q) dst[q] = v[q];
            }
        }
    }
    if (a.l1.w == 0) return;
    // Each horizontal mean once (every source row, 65 columns), then the
    // vertical pass; the same for the level after. Values computed outside
    // a level's size are never stored and only feed other such values.
    for (int i = tid; i < kSY * kS1X; i += kNT) {
        const int r = i / kS1X, c = i - r * kS1X;
        const float* p = &s0[r * kSXA + 2 * c];
        h1[i] = mean121(p[0], p[1], p[2]);
    }
    __syncthreads();
    const int x1 = x0 / 2, y1 = y0 / 2;
    for (int i = tid; i < kS1X * kS1Y; i += kNT) {
        const int r = i / kS1X, c = i - r * kS1X, x = x1 + c, y = y1 + r;
        const float* p = &h1[(2 * r) * kS1X + c];
        const float v = __fmul_rn(0.5f, mean121(p[0], p[kS1X], p[2 * kS1X]));
        if (x < a.l1.w && y < a.l1.h && c < kTX / 2 && r < kTY / 2) row_of(a.l1, a.pitch, y)[x] = v;
        s1[i] = v;
    }
    if (a.l2.w == 0) return;
    __syncthreads();
    for (int i = tid; i < kS1Y * (kTX / 4); i += kNT) {
        const int r = i / (kTX / 4), c = i - r * (kTX / 4);
        const float* p = &s1[r * kS1X + 2 * c];
        h2[i] = mean121(p[0], p[1], p[2]);
    }
    __syncthreads();
    {
        const int r = tid / (kTX / 4), c = tid % (kTX / 4), x = x0 / 4 + c, y = y0 / 4 + r;
        const float* p = &h2[(2 * r) * (kTX / 4) + c];
        if (x < a.l2.w && y < a.l2.h)
            row_of(a.l2, a.pitch, y)[x] = __fmul_rn(0.5f, mean121(p[0], p[kTX / 4], p[2 * (kTX / 4)]));
    }
}
static_assert((kTX / 4) * (kTY / 4) == kNT, "one thread per pixel of the second level");

// Levels first .. last from level first - 1, all in one CTA: the source
// level is staged in shared memory and each level is computed from the one
// before there (ping-pong buffers of kTailA and kTailB floats) and stored.
struct TailArgs {
    Level lv[32];
    int first, last;
    size_t pitch;
};

__global__ void __launch_bounds__(kTailThreads) tail_kernel(TailArgs a) {  // blockDim = kTailThreads
    __shared__ float buf[kTailA + kTailB];
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const Level s = a.lv[a.first - 1];
    float* cur = buf;
    float* nxt = buf + kTailA;
    stage<float, kTailThreads, kTailChunks>(cur, s.w, reinterpret_cast<const char*>(s.ptr), a.pitch, s.w,
                                                 s.h, 0, 0, s.w, s.h);
    __syncthreads();
    int cw = s.w;
    for (int k = a.first; k <= a.last; ++k) {
        const Level d = a.lv[k];
        for (int i = threadIdx.x; i < d.w * d.h; i += blockDim.x) {
            const int y = i / d.w, x = i - y * d.w;
            const float v = reduce3x3(&cur[(2 * y) * cw + 2 * x], cw);
            nxt[i] = v;
            row_of(d, a.pitch, y)[x] = v;
        }
        __syncthreads();
        float* t = cur;
        cur = nxt;
        nxt = t;
        cw = d.w;
    }
}

// Level geometry of a W x H packed mip-map: origin and size of each level
// 0 .. max_levels (level max_levels is the last non-empty one).
struct Geometry {
    int x1, max_levels;
    int x[32], y[32], w[32], h[32];
};

inline Geometry geometry(int W, int H) {
    Geometry g{};
    g.x1 = (W + 3) / 4 * 4;
    g.x[0] = g.y[0] = 0;
    g.w[0] = W;
    g.h[0] = H;
    int k = 0, yy = 0;
    while (k + 1 < 32 && next_size(g.w[k]) > 0 && next_size(g.h[k]) > 0) {
        g.w[k + 1] = next_size(g.w[k]);
        g.h[k + 1] = next_size(g.h[k]);
        g.x[k + 1] = g.x1;
        g.y[k + 1] = yy;
        yy += g.h[k + 1];
        ++k;
    }
    g.max_levels = k;
    return g;
}

inline cudaLaunchConfig_t chained(dim3 grid, dim3 block, cudaStream_t s, cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.stream = s;
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

}  // namespace mip
}  // namespace ct

using namespace ct;

extern "C" {

int ct_disp_mipmap_format(int32_t width, int32_t height, int32_t* packed_width, int32_t* max_levels) {
    clear_error();
    if (width <= 0 || height <= 0) return fail(CT_EINVAL, "bad size %dx%d", width, height);
    const mip::Geometry g = mip::geometry(width, height);
    if (packed_width) *packed_width = g.x1 + mip::next_size(width);
    if (max_levels) *max_levels = g.max_levels;
    return CT_OK;
}

int ct_disp_mipmap_level(int32_t width, int32_t height, int32_t level, int32_t* x, int32_t* y, int32_t* w,
                         int32_t* h) {
    clear_error();
    if (width <= 0 || height <= 0) return fail(CT_EINVAL, "bad size %dx%d", width, height);
    const mip::Geometry g = mip::geometry(width, height);
    if (level < 0 || level > g.max_levels)
        return fail(CT_EINVAL, "level %d outside 0 .. %d", level, g.max_levels);
    if (x) *x = g.x[level];
    if (y) *y = g.y[level];
    if (w) *w = g.w[level];
    if (h) *h = g.h[level];
    return CT_OK;
}

int ct_disp_mipmaps(const ct_image* mipmap, const ct_image* disp, int32_t level_count, ct_stream stream) {
    clear_error();
    if (int rc = check_image(disp, "disp", (1u << CT_PIX_U8) | (1u << CT_PIX_U16))) return rc;
    if (int rc = check_image(mipmap, "mipmap", 1u << CT_PIX_F32)) return rc;
    const int W = disp->width, H = disp->height;
    const mip::Geometry g = mip::geometry(W, H);
    const int pw = g.x1 + mip::next_size(W);
    if (mipmap->width != pw || mipmap->height != H)
        return fail(CT_EFORMAT, "mipmap is %dx%d; a %dx%d disparity map needs %dx%d", mipmap->width,
                    mipmap->height, W, H, pw, H);
    // CDriver::Run's level count rules (CreateDispMipMaps.cu:268-282): more
    // than the maximum is an error, <= 0 means the maximum, 1 does nothing;
    // levels 0 .. count - 1 are written.
    if (level_count > g.max_levels)
        return fail(CT_EINVAL, "level count %d larger than the maximal possible level count %d", level_count,
                    g.max_levels);
    if (level_count <= 0) level_count = g.max_levels;
    else if (level_count == 1) return CT_OK;
    const int last = level_count > 1 ? level_count - 1 : 0;  // highest level written

    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const size_t pitch = mipmap->pitch_bytes;
    auto level = [&](int k) {
        char* p = static_cast<char*>(mipmap->ptr) + (size_t)g.y[k] * pitch + (size_t)g.x[k] * sizeof(float);
        return mip::Level{reinterpret_cast<float*>(p), g.w[k], g.h[k]};
    };
    const mip::Level none{nullptr, 0, 0};
    cudaLaunchAttribute attr[1];
    // levels 0 .. min(last, 2) from the code map
    {
        mip::FusedArgs fa{disp->ptr, disp->pitch_bytes, W, H, level(0), last >= 1 ? level(1) : none,
                          last >= 2 ? level(2) : none, pitch};
        cudaLaunchConfig_t cfg = mip::chained(dim3((W + mip::kTX - 1) / mip::kTX, (H + mip::kTY - 1) / mip::kTY),
                                              dim3(mip::kNT), s, attr);
        if (disp->type == CT_PIX_U8)
            CT_CUDA_TRY(cudaLaunchKernelEx(&cfg, mip::fused_kernel<uint8_t>, fa));
        else
            CT_CUDA_TRY(cudaLaunchKernelEx(&cfg, mip::fused_kernel<uint16_t>, fa));
    }
    int done = last < 2 ? last : 2;  // highest level written so far
    while (done < last) {
        const mip::Level src = level(done);
        if (src.w * src.h <= mip::kTailA && (src.w + 3) / 4 * src.h <= mip::kTailChunks) {
            // every remaining level from shared memory
            mip::TailArgs ta{};
            for (int i = 0; i <= last; ++i) ta.lv[i] = level(i);
            ta.first = done + 1;
            ta.last = last;
            ta.pitch = pitch;
            cudaLaunchConfig_t cfg = mip::chained(dim3(1), dim3(mip::kTailThreads), s, attr);
            CT_CUDA_TRY(cudaLaunchKernelEx(&cfg, mip::tail_kernel, ta));
            break;
        }
        mip::FusedArgs fa{src.ptr, pitch, src.w, src.h, none, level(done + 1),
                          done + 2 <= last ? level(done + 2) : none, pitch};
        cudaLaunchConfig_t cfg = mip::chained(
            dim3((src.w + mip::kTX - 1) / mip::kTX, (src.h + mip::kTY - 1) / mip::kTY), dim3(mip::kNT), s, attr);
        CT_CUDA_TRY(cudaLaunchKernelEx(&cfg, mip::fused_kernel<float>, fa));
        done = done + 2 <= last ? done + 2 : last;
    }
    CT_LAUNCH_CHECK();
    return CT_OK;
}

}  // extern "C"
