// confnet.cu — learned confidence for census disparities: a small 1D-conv +
// MLP network that reads a pixel's census cost curve (128 disparities, one
// byte each, from ct_bm_census_process_curves) and scores how likely the
// winner-take-all disparity is correct. It stands in for the right-to-left
// matching pass of the left-right check (CrossCheckDisparityMaps.cu:63-110),
// which stays as the fallback and as the yardstick for its error.
//
// Network (weights bf16, biases fp32, accumulation fp32):
//   input  the pixel's curve re-centred on its winning disparity d: sample
//          r[k] = c[d - 64 + k] (255 outside); the convolutions read the 35
//          codes x[k] = r[52 + k] (disparities d - 12 .. d + 22)
//   conv1  1 -> 32, k=5, stride 5 -> 7 positions; ReLU; bf16 -> a1[7][32]
//   conv2 32 -> 32, k=5, stride 3, pad 1 -> 2 positions; ReLU; bf16 -> a2[2][32]
//   conv3 32 -> 32, k=5, pad 2, one output (taps 2, 3 meet data); ReLU; bf16 -> a3[32]
//   fc1   32 -> 64, ReLU (fp32) -> a4[64]
//   fc2   64 -> 1, logit; score = sigmoid(logit)
// Flat parameter order: w1[32][5], b1[32], w2[32][32][5] ([out][in][tap]),
// b2[32], w3[32][32][5], b3[32], w4[64][32], b4[64], w5[64], b5[1].
//
// Training: the dense layers (conv2, conv3, fc1: forward, data gradients
// and weight gradients) are bf16 GEMMs with fp32 accumulation on the tensor
// cores (tg::gemm_kernel); conv1, the head and the elementwise steps (bias,
// ReLU, bf16 rounding, masks) run on the CUDA cores with one thread per
// (sample, channel). Weight gradients are reduced per chunk of samples into
// partial sums that the Adam kernel adds in a fixed order (deterministic).
// Adam keeps fp32 master weights and writes their bf16 roundings for the
// next forward.
//
// Inference (tensor cores, tcgen05): a persistent kernel of one warpgroup per
// CTA, two CTAs per SM, 128 pixels (a row segment) per tile = the M of every
// MMA. conv1 is three MMAs over an im2col of the 35 codes (15 per K=16
// window, f16: the codes are integers and the bf16 weights are exact in
// f16); conv2, conv3 and fc1 read their activations from tensor memory (the
// A-from-TMEM form) and bf16 weights from shared memory. Biases are written
// into the fp32 accumulator columns with tcgen05.st before each layer; the
// epilogues read them with tcgen05.ld, apply ReLU, round to bf16 and store
// the next layer's A operand back into the tensor memory they have consumed.
// Each tile's block of curve words (all disparity groups of its 128 columns)
// arrives by one TMA load issued a tile ahead; the disparity entries are read
// two tiles ahead, so no thread waits on a global load inside the loop.
#include "ct_internal.h"
#include "ct_device.cuh"
#include "census_match.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cmath>
#include <cstring>
#include <vector>

namespace ct {
namespace cn {

// ---------------------------------------------------------------------------
// Parameter layout
// ---------------------------------------------------------------------------
constexpr int kOffW1 = 0, kOffB1 = 160, kOffW2 = 192, kOffB2 = 5312, kOffW3 = 5344, kOffB3 = 10464,
              kOffW4 = 10496, kOffB4 = 12544, kOffW5 = 12608, kOffB5 = 12672;
constexpr int kParams = 12673;
static_assert(kParams == CT_CONFNET_PARAMS, "parameter count");
constexpr int kLen = 128;  // curve length (disparities)
constexpr int kCropLo = 52, kCropLen = 35;  // codes of the re-centred sample the convolutions read

__host__ __device__ inline bool is_weight(int p) {
    return p < kOffB1 || (p >= kOffW2 && p < kOffB2) || (p >= kOffW3 && p < kOffB3) || (p >= kOffW4 && p < kOffB4) ||
           (p >= kOffW5 && p < kOffB5);
}

__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }
__device__ __forceinline__ uint16_t bf16_bits(float v) { return __bfloat16_as_ushort(__float2bfloat16_rn(v)); }

// ---------------------------------------------------------------------------
// Gather: samples[n][128] from a curve volume at pixel list xy[n][2]
// ---------------------------------------------------------------------------
// A disparity map entry as stored (U8 or U16).
__device__ __forceinline__ uint32_t disp_entry(const void* disp, size_t pitch, int type, int x, int y) {
    const char* row = static_cast<const char*>(disp) + (size_t)y * pitch;
    return type == CT_PIX_U8 ? uint32_t(reinterpret_cast<const uint8_t*>(row)[x])
                             : uint32_t(reinterpret_cast<const uint16_t*>(row)[x]);
}
// Winning disparity of a map entry (U16 EDisparityId d + 1, U8 d; 0 when the
// pixel has no disparity).
__device__ __forceinline__ int entry_winner(uint32_t v, int type) {
    if (type == CT_PIX_U8) return v < uint32_t(kLen) ? int(v) : 0;
    return (v >= 1 && v <= uint32_t(kLen)) ? int(v) - 1 : 0;
}
__device__ __forceinline__ int winner(const void* disp, size_t pitch, int type, int x, int y) {
    return entry_winner(disp_entry(disp, pitch, type, x, y), type);
}

// Re-centred samples: samples[s][k] = curve(x, y)[d - 64 + k] (255 outside),
// d the pixel's winning disparity. One warp per sample, lane = output word.
// Pixels outside the volume read as all-255 samples and set CT_EINVAL.
__global__ void gather_kernel(uint8_t* samples, const uint32_t* curve, size_t pitch_words, int W, int H,
                              const void* disp, size_t disp_pitch, int disp_type, const int32_t* xy, int n,
                              int32_t* status) {
    const int s = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (s >= n) return;
    const int x = xy[2 * s], y = xy[2 * s + 1];
    const bool inside = x >= 0 && x < W && y >= 0 && y < H;
    if (!inside && lane == 0) dev::report(status, CT_EINVAL);
    uint32_t w = 0xFFFFFFFFu;
    if (inside) {
        const int b0 = winner(disp, disp_pitch, disp_type, x, y) - 64 + 4 * lane;  // first curve byte of this word
        const int g0 = b0 >> 2, sh = (b0 & 3) * 8;                                 // arithmetic shift: floor
        auto word = [&](int g) {
            return (g >= 0 && g < kLen / 4) ? curve[((size_t)y * (kLen / 4) + g) * pitch_words + x + 2] : 0xFFFFFFFFu;
        };
        w = __funnelshift_r(word(g0), word(g0 + 1), sh);
    }
    reinterpret_cast<uint32_t*>(samples + (size_t)s * kLen)[lane] = w;
}

// ---------------------------------------------------------------------------
// Training kernels (block (32, 16): threadIdx.x = channel, threadIdx.y = sample)
// ---------------------------------------------------------------------------
struct Act {  // per-sample activations and gradient signals, [n][...]
    float* a1;      // [7][32] bf16 values
    float* a2;      // [2][32]
    float* a3;      // [32]
    float* a4;      // [64]
    float* logit;   // [1]
    float* dl;      // dloss/dlogit
    float* loss;    // per-sample loss
    float* dz4;     // [64]
    float* dz3;     // [32]
    float* dz2;     // [2][32]
    float* dm1;     // [7][32]
    // bf16 operands of the tensor-core GEMMs (tg::gemm_kernel): row-major
    // [n][features] and transposed [features][ldt] (samples contiguous;
    // columns n .. n rounded up to 8 hold 0)
    uint16_t *a1p, *a1pt;  // [n][256]: slot 0 = 0, slots 1..7 = conv1 positions 0..6; [256][ldt]
    uint16_t *a2b, *a2t, *a3b, *a3t;
    uint16_t *dz4b, *dz4t, *dz3b, *dz3t, *dz2b, *dz2t;
    float* d;              // GEMM output scratch [n][224]
    int ldt;
};
constexpr int kQ = 7;   // pooled conv1 positions
constexpr int kR = 2;   // conv2 positions

constexpr int kSY = 16;  // samples per CTA

// conv1 (k=5, stride 5) over the 35 central codes, ReLU, bf16; also the
// bf16 operand copies of the conv2 GEMMs (forward and weight gradient)
__global__ void __launch_bounds__(32 * kSY) fwd1_kernel(const uint8_t* x, const float* wq, Act A, int n) {
    __shared__ float xs[kSY][kLen];
    const int o = threadIdx.x, sl = threadIdx.y, s = blockIdx.x * kSY + sl;
    for (int k = threadIdx.x; k < kLen; k += 32) xs[sl][k] = s < n ? float(x[(size_t)s * kLen + k]) : 0.f;
    __syncthreads();
    if (s >= ((n + 7) & ~7)) return;
    if (s >= n) {  // transposed columns past n read as 0
#pragma unroll
        for (int q = 0; q <= kQ; ++q) A.a1pt[(size_t)(q * 32 + o) * A.ldt + s] = 0;
        return;
    }
    float w[5];
#pragma unroll
    for (int j = 0; j < 5; ++j) w[j] = wq[kOffW1 + o * 5 + j];
    const float b = wq[kOffB1 + o];
    A.a1p[(size_t)s * 256 + o] = 0;
    A.a1pt[(size_t)o * A.ldt + s] = 0;
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
        float z = b;
#pragma unroll
        for (int j = 0; j < 5; ++j) z = fmaf(w[j], xs[sl][kCropLo + 5 * q + j], z);
        const float v = bf16r(fmaxf(z, 0.f));
        A.a1[(size_t)s * 224 + q * 32 + o] = v;
        const uint16_t vb = bf16_bits(v);
        A.a1p[(size_t)s * 256 + (q + 1) * 32 + o] = vb;
        A.a1pt[(size_t)((q + 1) * 32 + o) * A.ldt + s] = vb;
    }
}

// Epilogue of a forward GEMM (block (32, 8), 8 samples): v = ReLU(d + bias)
// (bias[col % bmod]; rounded to bf16 when rnd) into f [n][N] and the bf16
// operand copies b [n][N] and t [N][ldt] when given.
__global__ void ep_fwd_kernel(const float* d, int N, const float* bias, int bmod, int rnd, float* f, uint16_t* b,
                              uint16_t* t, int ldt, int n) {
    const int s = blockIdx.x * 8 + threadIdx.y;
    if (s >= ((n + 7) & ~7)) return;
    for (int c = threadIdx.x; c < N; c += 32) {
        if (s >= n) {
            if (t) t[(size_t)c * ldt + s] = 0;
            continue;
        }
        float v = fmaxf(d[(size_t)s * N + c] + bias[c % bmod], 0.f);
        if (rnd) v = bf16r(v);
        f[(size_t)s * N + c] = v;
        if (b) b[(size_t)s * N + c] = bf16_bits(v);
        if (t) t[(size_t)c * ldt + s] = bf16_bits(v);
    }
}

// Epilogue of a data-gradient GEMM (block (32, 8)): g = act > 0 ? d : 0 into
// f [n][N] and the bf16 copies b, t when given.
__global__ void ep_bwd_kernel(const float* d, int N, const float* act, float* f, uint16_t* b, uint16_t* t, int ldt,
                              int n) {
    const int s = blockIdx.x * 8 + threadIdx.y;
    if (s >= ((n + 7) & ~7)) return;
    for (int c = threadIdx.x; c < N; c += 32) {
        if (s >= n) {
            if (t) t[(size_t)c * ldt + s] = 0;
            continue;
        }
        const size_t k = (size_t)s * N + c;
        const float g = act[k] > 0.f ? d[k] : 0.f;
        f[k] = g;
        if (b) b[k] = bf16_bits(g);
        if (t) t[(size_t)c * ldt + s] = bf16_bits(g);
    }
}

// one thread per sample: logit, loss, dloss/dlogit (labels may be null: scores only)
__global__ void head_kernel(const float* wq, Act A, const uint8_t* labels, float inv_n, float* scores, int n) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float z = wq[kOffB5];
    for (int h = 0; h < 64; ++h) z = fmaf(wq[kOffW5 + h], A.a4[(size_t)s * 64 + h], z);
    A.logit[s] = z;
    const float p = 1.f / (1.f + expf(-z));
    if (scores) scores[s] = p;
    if (labels) {
        const float y = labels[s] ? 1.f : 0.f;
        A.dl[s] = (p - y) * inv_n;
        A.loss[s] = fmaxf(z, 0.f) + log1pf(expf(-fabsf(z))) - y * z;
    }
}

// block (64, 8): dz4 = dl * w5 * (a4 > 0), with its bf16 operand copies
__global__ void bwd4_kernel(const float* wq, Act A, int n) {
    const int h = threadIdx.x, s = blockIdx.x * 8 + threadIdx.y;
    if (s >= ((n + 7) & ~7)) return;
    if (s >= n) {
        A.dz4t[(size_t)h * A.ldt + s] = 0;
        return;
    }
    const float a = A.a4[(size_t)s * 64 + h];
    const float g = a > 0.f ? A.dl[s] * wq[kOffW5 + h] : 0.f;
    A.dz4[(size_t)s * 64 + h] = g;
    A.dz4b[(size_t)s * 64 + h] = bf16_bits(g);
    A.dz4t[(size_t)h * A.ldt + s] = bf16_bits(g);
}

// Weight gradients of one chunk of samples (blockIdx.x) on the CUDA cores,
// written to part[chunk][param]: conv1 (blockIdx.y 0), the biases of conv2,
// conv3 and fc1 (1, 2, 3; their weights come from the tensor-core GEMMs)
// and fc2 (4). 256 threads.
constexpr int kChunk = 256;

__global__ void __launch_bounds__(256) wgrad_kernel(const uint8_t* x, Act A, int n, float* part) {
    const int t = threadIdx.x;
    const int s0 = blockIdx.x * kChunk, s1 = min(n, s0 + kChunk);
    float* P = part + (size_t)blockIdx.x * kParams;
    switch (blockIdx.y) {
        case 0: {  // w1 (o, j) for t < 160, b1 for 160 <= t < 192
            if (t >= 192) return;
            const bool bias = t >= 160;
            const int o = bias ? t - 160 : t / 5, j = t % 5;
            float acc = 0.f;
            for (int s = s0; s < s1; ++s) {
                for (int q = 0; q < kQ; ++q) {
                    const float g = A.dm1[(size_t)s * 224 + q * 32 + o];
                    if (g == 0.f) continue;
                    if (bias) { acc += g; continue; }
                    acc = fmaf(g, float(x[(size_t)s * kLen + kCropLo + 5 * q + j]), acc);
                }
            }
            P[bias ? kOffB1 + o : kOffW1 + t] = acc;
            break;
        }
        case 1: {  // b2 (w2 by the tensor-core GEMM, tg::kW2T)
            if (t >= 32) return;
            float bacc = 0.f;
            for (int s = s0; s < s1; ++s)
                for (int r = 0; r < kR; ++r) bacc += A.dz2[(size_t)s * 64 + r * 32 + t];
            P[kOffB2 + t] = bacc;
            break;
        }
        case 2: {  // b3, and 0 for the taps of w3 that meet no data (taps 2, 3 by tg::kW3T)
            for (int k = t; k < 32 * 32 * 3; k += 256) {
                const int oi = k / 3, j = k % 3;
                P[kOffW3 + oi * 5 + (j == 2 ? 4 : j)] = 0.f;
            }
            if (t >= 32) return;
            float bacc = 0.f;
            for (int s = s0; s < s1; ++s) bacc += A.dz3[(size_t)s * 32 + t];
            P[kOffB3 + t] = bacc;
            break;
        }
        case 3: {  // b4 (w4 by tg::kW4)
            if (t >= 64) return;
            float bacc = 0.f;
            for (int s = s0; s < s1; ++s) bacc += A.dz4[(size_t)s * 64 + t];
            P[kOffB4 + t] = bacc;
            break;
        }
        default: {  // w5 for t < 64, b5 for t == 64
            if (t > 64) return;
            float acc = 0.f;
            for (int s = s0; s < s1; ++s) acc += t < 64 ? A.dl[s] * A.a4[(size_t)s * 64 + t] : A.dl[s];
            P[t < 64 ? kOffW5 + t : kOffB5] = acc;
            break;
        }
    }
}

// Sums the chunk partials (fixed order) into grad; with adam != 0 also
// applies one Adam step to the fp32 master weights and refreshes wq.
struct AdamArgs {
    int adam;
    float lr, beta1, beta2, eps, c1, c2;  // c1 = 1 - beta1^t, c2 = 1 - beta2^t
};

__global__ void reduce_adam_kernel(const float* part, int chunks, float* grad, float* master, float* m, float* v,
                                   float* wq, AdamArgs aa) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    float g = 0.f;
    for (int c = 0; c < chunks; ++c) g += part[(size_t)c * kParams + p];
    if (grad) grad[p] = g;
    if (!aa.adam) return;
    const float mm = aa.beta1 * m[p] + (1.f - aa.beta1) * g;
    const float vv = aa.beta2 * v[p] + (1.f - aa.beta2) * g * g;
    m[p] = mm;
    v[p] = vv;
    const float w = master[p] - aa.lr * (mm / aa.c1) / (sqrtf(vv / aa.c2) + aa.eps);
    master[p] = w;
    wq[p] = is_weight(p) ? bf16r(w) : w;
}

// Deterministic mean of the per-sample losses (one CTA).
__global__ void loss_mean_kernel(const float* loss, int n, float* out) {
    __shared__ float red[256];
    float acc = 0.f;
    for (int s = threadIdx.x; s < n; s += 256) acc += loss[s];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = red[0] / float(n);
}

// ---------------------------------------------------------------------------
// Inference kernel (tcgen05)
// ---------------------------------------------------------------------------
namespace inf {

constexpr int kNT = 128;  // one warpgroup: thread = pixel of the tile = TMEM lane
constexpr int kM = 128;   // pixels per tile = MMA M
constexpr int kChunkBytes = kM * 16;  // one K-chunk (8 elements) of the 128-row A1 operand

// Shared memory:
//   box    the tile's curve block, brought in by one TMA load: all 32
//          disparity groups x kBoxWords words starting at word x0 (the tile's
//          first column x0 is word x0 + 2), group g at g * kBoxWords words;
//          pixel m reads column m + 2 (lanes of a warp on distinct banks
//          when they share the group)
//   A1     conv1 operand, f16, K-major without swizzle in K-chunk panels
//          (element (pixel r, k) at (k / 8) * 2048 + r * 16 + (k % 8) * 2):
//          window t = chunks 2t, 2t + 1 holds codes 15t .. 15t + 15 of the
//          35 the convolutions read (codes past the 35th meet zero weights)
//   then the packed weights (B operands in the same panel form with rows =
//   output channels, and fp32 biases).
constexpr int kGroups = 32;       // 128 disparities / 4 per word
constexpr int kBoxWords = kM + 4; // 2 halo words + 128 columns, rounded to 16 bytes
constexpr int kBoxBytes = kGroups * kBoxWords * 4;
constexpr int kBox = 0;
constexpr int kA1 = kBox + kBoxBytes;
constexpr int kA1Chunks = 6;
constexpr int kWImg = kA1 + kA1Chunks * kChunkBytes;
constexpr int kB1 = 0;                  // conv1: N=96 (position-in-window x 32) x K=16 f16, tap j of
                                        // window position pp at k = 5 pp + j (LBO 96 * 16)
constexpr int kB2 = kB1 + 2 * 1536;     // conv2: N=32 x K=160 bf16, chunk = tap * 4 + in / 8 (LBO 512)
constexpr int kB3 = kB2 + 20 * 512;     // conv3 taps 2, 3: N=32 x K=64, chunk = (tap - 2) * 4 + in / 8
constexpr int kB4 = kB3 + 8 * 512;      // fc1: N=64 x K=32 bf16 (LBO 1024)
constexpr int kBias = kB4 + 4 * 1024;   // fp32: b1[32] b2[32] b3[32] b4[64] w5[64] b5
constexpr int kWBytes = kBias + (32 + 32 + 32 + 64 + 64 + 4) * 4;
constexpr int kBar = kWImg + kWBytes;   // 3 mbarriers: MMA commits (2), curve block
constexpr int kTmemSlot = kBar + 3 * 8;
constexpr int kSmem = kTmemSlot + 16;
static_assert(kWBytes % 16 == 0, "weight image must be a whole number of 16-byte words");
static_assert(kBoxWords * 4 % 16 == 0 && kA1 % 128 == 0, "TMA box rows and A1 panels 16-byte aligned");
static_assert(2 * kSmem <= 228 * 1024, "two CTAs per SM");

// TMEM (256 columns per CTA, two CTAs per SM). Accumulators are fp32, one
// column per output; A operands held in TMEM are bf16 pairs, a K=16 slice =
// 8 columns. Regions are reused as soon as what they held has been read:
//   C1 conv1 accumulators, position q at 32 q                  0 .. 223
//   A2 conv1 output (bf16), position q at 16 q                0 .. 111
//   C2 conv2 accumulators, position r at 128 + 32 r          128 .. 191
//   A3 conv2 output, position r at 192 + 16 r                192 .. 223
//   C3 conv3 accumulators                                      0 .. 31
//   A4 conv3 output                                           32 .. 47
//   C4 fc1 accumulators                                       64 .. 127
constexpr uint32_t kTmemCols = 256;
constexpr uint32_t kC2 = 128, kA3 = 192, kC3 = 0, kA4 = 32, kC4 = 64;

// Instruction descriptors (kind::f16): D fp32 (bit 4), A/B format at bits
// 7 / 10 (0 = f16, 1 = bf16), both K-major, N >> 3 at bit 17, M >> 4 at 24.
constexpr uint32_t idesc(int fmt, int N) {
    return (1u << 4) | (uint32_t(fmt) << 7) | (uint32_t(fmt) << 10) | (uint32_t(N >> 3) << 17) |
           (uint32_t(kM >> 4) << 24);
}
constexpr uint32_t kIdC1 = idesc(0, 96), kIdC1n = idesc(0, 32), kIdC2 = idesc(1, 32), kIdF1 = idesc(1, 64);

// Shared-memory matrix descriptor: start, leading byte offset (next K chunk),
// stride byte offset 128 (next 8 rows), version 1, no swizzle.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo) {
    return uint64_t((saddr >> 4) & 0x3FFF) | (uint64_t((lbo >> 4) & 0x3FFF) << 16) | (uint64_t(128 >> 4) << 32) |
           (uint64_t(1) << 46);
}

// A descriptor moved by `bytes` (a multiple of 16) along its start field.
__device__ __forceinline__ uint64_t dplus(uint64_t d, uint32_t bytes) { return d + uint64_t(bytes >> 4); }

// The MMA helpers are executed by a whole (converged) warp; one elected lane
// issues. Warp-uniform operands stay in uniform registers, which makes the
// issue of consecutive MMAs several times cheaper than from a lone thread.
// D (TMEM) += A (shared memory) x B (shared memory)
__device__ __forceinline__ void mma_ss(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t id) {
    asm volatile(
        "{\n.reg .pred p, e;\nsetp.ne.b32 p, 1, 0;\nelect.sync _|e, 0xffffffff;\n"
        "@e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(id)
        : "memory");
}
// D (TMEM) += A (TMEM, lane = row, K packed in pairs per column) x B (shared memory)
__device__ __forceinline__ void mma_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t b, uint32_t id) {
    asm volatile(
        "{\n.reg .pred p, e;\nsetp.ne.b32 p, 1, 0;\nelect.sync _|e, 0xffffffff;\n"
        "@e tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n}\n" ::"r"(tmem_d),
        "r"(tmem_a), "l"(b), "r"(id)
        : "memory");
}
// Completion of this warp's MMAs so far -> one arrive on bar (elected lane).
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile(
        "{\n.reg .pred e;\nelect.sync _|e, 0xffffffff;\n"
        "@e tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n}\n" ::"r"(
            dev::smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// 32 consecutive TMEM columns of this thread's lane, with the load's wait in
// the same asm statement (the registers are defined only after completion).
__device__ __forceinline__ void ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "{\n"
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        "}\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int k = 0; k < 32; ++k) v[k] = __uint_as_float(r[k]);
}
// Two 32-column loads (columns taddr .. +31 and taddr2 .. +31), one wait.
__device__ __forceinline__ void ld32x2(uint32_t taddr, uint32_t taddr2, float (&v)[32], float (&u)[32]) {
    uint32_t r[64];
    asm volatile(
        "{\n"
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%64];\n"
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47,%48,%49,%50,%51,%52,%53,%54,%55,%56,%57,%58,%59,%60,%61,%62,%63}, [%65];\n"
        "tcgen05.wait::ld.sync.aligned;\n"
        "}\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]), "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]), "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]), "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]), "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr), "r"(taddr2)
        : "memory");
#pragma unroll
    for (int k = 0; k < 32; ++k) {
        v[k] = __uint_as_float(r[k]);
        u[k] = __uint_as_float(r[32 + k]);
    }
}
__device__ __forceinline__ void st32(uint32_t taddr, const float (&v)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
        "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
        "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
        "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])),
        "r"(__float_as_uint(v[11])), "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])),
        "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15])), "r"(__float_as_uint(v[16])),
        "r"(__float_as_uint(v[17])), "r"(__float_as_uint(v[18])), "r"(__float_as_uint(v[19])),
        "r"(__float_as_uint(v[20])), "r"(__float_as_uint(v[21])), "r"(__float_as_uint(v[22])),
        "r"(__float_as_uint(v[23])), "r"(__float_as_uint(v[24])), "r"(__float_as_uint(v[25])),
        "r"(__float_as_uint(v[26])), "r"(__float_as_uint(v[27])), "r"(__float_as_uint(v[28])),
        "r"(__float_as_uint(v[29])), "r"(__float_as_uint(v[30])), "r"(__float_as_uint(v[31]))
        : "memory");
}
__device__ __forceinline__ void st16(uint32_t taddr, const uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
            taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
        "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
        : "memory");
}

// bf16x2 with relu: low half = a, high half = b
__device__ __forceinline__ uint32_t pack_relu(float a, float b) {
    uint32_t d;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(b), "f"(a));
    return d;
}
// Two curve codes (bytes sel of w) -> f16x2 of their integer values: the
// bytes become the low mantissa of 1024.0 (0x6400), then 1024 is subtracted.
__device__ __forceinline__ uint32_t codes_f16x2(uint32_t w, uint32_t sel) {
    const uint32_t h = __byte_perm(w, 0x64646464u, sel);
    uint32_t d;
    asm("sub.rn.f16x2 %0, %1, %2;" : "=r"(d) : "r"(h), "r"(0x64006400u));
    return d;
}
// 32 accumulators -> ReLU -> bf16 pairs -> 16 TMEM columns (an A operand row)
__device__ __forceinline__ void relu_bf16_to_tmem(uint32_t dst, const float (&v)[32]) {
    uint32_t o[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) o[c] = pack_relu(v[2 * c], v[2 * c + 1]);
    st16(dst, o);
}

struct InferArgs {
    const uint32_t* curve;
    size_t curve_pitch;  // words
    int groups;          // 32
    const void* disp;    // winning disparities (U8 or U16 map)
    size_t disp_pitch;
    int disp_type;
    int W, H;
    float* score;        // may be null
    size_t score_pitch;  // bytes
    void* checked;       // may be null: the winner map with rejected pixels marked
    size_t checked_pitch;
    float threshold;
    const uint4* wimg;   // packed weight image (kWBytes)
    int32_t* status;
};

__global__ void __launch_bounds__(kNT, 2) infer_kernel(const __grid_constant__ CUtensorMap tm_curve, InferArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int m = tid;  // pixel of the tile / TMEM lane
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + kBar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kTmemSlot);
    unsigned char* A1 = smem + kA1;
    const uint32_t* box = reinterpret_cast<const uint32_t*>(smem + kBox) + m + 2;  // this pixel's column
    const uint32_t sA1 = dev::smem_u32(A1), sW = dev::smem_u32(smem + kWImg);

    for (int k = tid; k < kWBytes / 16; k += kNT) reinterpret_cast<uint4*>(smem + kWImg)[k] = a.wimg[k];
    if (tid == 0) {
        dev::mbar_init(&bars[0], 1);
        dev::mbar_init(&bars[1], 1);
        dev::mbar_init(&bars[2], 1);
        dev::fence_barrier_init();
        dev::prefetch_tmap(&tm_curve);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dev::smem_u32(tslot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tm = *tslot;
    const uint32_t tl = tm + (uint32_t(warp * 32) << 16);  // this warp's lane quarter
    // Launched with programmatic stream serialisation, this kernel may start
    // while the matcher that writes the curves and winners is still running:
    // everything above reads only the weight image; wait here for the
    // previous grid's results before the first curve or disparity read.
    asm volatile("griddepcontrol.wait;" ::: "memory");

    const float* bias = reinterpret_cast<const float*>(smem + kWImg + kBias);
    const float* w5 = bias + 160;
    static_assert((kWImg + kBias + 160 * 4) % 16 == 0, "w5 is read as float4");
    const float b5 = bias[224];
    float bias1[32];  // conv1 biases, stored into 7 accumulator groups per tile
#pragma unroll
    for (int c = 0; c < 32; ++c) bias1[c] = bias[c];
    // base descriptors; every operand of a tile is a constant offset from one
    const uint64_t dA1 = sdesc(sA1, kChunkBytes);
    const uint64_t dB1 = sdesc(sW + kB1, 1536);
    const uint64_t dB2 = sdesc(sW + kB2, 512), dB3 = sdesc(sW + kB3, 512), dB4 = sdesc(sW + kB4, 1024);

    const int tiles_x = (a.W + kM - 1) / kM;
    const int tiles = tiles_x * a.H;
    // Tile t = (row t / tiles_x, column tile t % tiles_x). A CTA visits tiles
    // t, t + G, ... (G = gridDim.x) and tracks three of them ahead by adding
    // (G / tiles_x, G % tiles_x) with a carry, never dividing in the loop.
    struct TilePos {
        int y, tx;
    };
    const int step_y = (int)gridDim.x / tiles_x, step_x = (int)gridDim.x % tiles_x;
    auto advance = [&](TilePos q) {
        q.y += step_y;
        q.tx += step_x;
        if (q.tx >= tiles_x) {
            q.tx -= tiles_x;
            ++q.y;
        }
        return q;
    };
    uint32_t ph[3] = {0, 0, 0};  // phases waited for, per mbarrier
    uint32_t cm[3] = {0, 0, 0};  // commits / loads issued (counted by the issuing warp's lanes)
    bool failed = false;
    auto commit_to = [&](int b) {
        commit(&bars[b]);
        ++cm[b];
    };
    auto wait_bar = [&](int b) {  // a phase that timed out stays pending in ph
        const bool ok = dev::mbar_wait_bounded(&bars[b], ph[b] & 1);
        if (ok) ++ph[b];
        return ok;
    };
    auto bias_to_tmem = [&](uint32_t col, const float* src) {  // src 16-byte aligned
        float bv[32];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const float4 q = reinterpret_cast<const float4*>(src)[c];
            bv[4 * c] = q.x;
            bv[4 * c + 1] = q.y;
            bv[4 * c + 2] = q.z;
            bv[4 * c + 3] = q.w;
        }
        st32(tl + col, bv);
    };
    // all threads: make this thread's TMEM / shared writes visible, then let
    // thread 0 issue the next MMAs
    auto hand_to_issuer = [&](bool smem_written) {
        wait_st();
        if (smem_written) dev::fence_proxy_async();
        fence_before();
        __syncthreads();
    };

    // A tile's disparity entries are loaded two tiles ahead and kept as
    // loaded (nothing consumes them before the next tile, so no thread waits
    // on the load); they give the curve offsets of the next tile's A1 and the
    // checked output without a second read of the map. The curve block of
    // the next tile is one TMA load, issued by lane 0 of warp 1 while the
    // conv1 MMAs run and waited for just before its A1 is built.
    auto load_entry = [&](TilePos q) {
        const int x = q.tx * kM + m;
        return x < a.W ? disp_entry(a.disp, a.disp_pitch, a.disp_type, x, q.y) : 0u;
    };
    auto load_box = [&](TilePos q) {  // warp 1, all lanes (they count the loads)
        if ((tid & 31) == 0) {
            dev::mbar_arrive_expect_tx(&bars[2], kBoxBytes);
            dev::tma_load_3d(smem + kBox, &tm_curve, q.tx * kM, 0, q.y, &bars[2]);
        }
        ++cm[2];
    };

    // A1 of the tile whose curve block is in the box: the 35 codes around
    // the winner d (curve bytes d - 12 .. d + 22; 255 outside the curve),
    // 15 per K=16 window
    auto build_a1 = [&](int d) {
        const int g0 = (d - 12) >> 2;  // floor: word of the first code
        const int c0 = (d - 12) - 4 * g0;
        // words g0 .. g0 + 9 hold the 35 codes (bytes c0 .. c0 + 34); later
        // words only feed codes that meet zero weights, so they read 255
        uint32_t w[13];
#pragma unroll
        for (int k = 0; k < 10; ++k) {
            const int g = g0 + k;
            w[k] = unsigned(g) < unsigned(kGroups) ? box[g * kBoxWords] : 0xFFFFFFFFu;
        }
        w[10] = w[11] = w[12] = 0xFFFFFFFFu;
#pragma unroll
        for (int t3 = 0; t3 < 3; ++t3) {
            // codes b0 .. b0 + 15 start in word b0 / 4, one of two words per window
            const int b0 = c0 + 15 * t3, sh = (b0 & 3) * 8;
            const bool hi = t3 == 0 ? false : (t3 == 1 ? c0 >= 1 : c0 >= 2);
            constexpr int kLo[3] = {0, 3, 7};
            uint32_t v[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint32_t r0 = hi ? w[kLo[t3] + k + 1] : w[kLo[t3] + k];
                const uint32_t r1 = hi ? w[kLo[t3] + k + 2] : w[kLo[t3] + k + 1];
                v[k] = __funnelshift_r(r0, r1, sh);
            }
            unsigned char* dst = A1 + 2 * t3 * kChunkBytes + m * 16;
            *reinterpret_cast<uint4*>(dst) = make_uint4(codes_f16x2(v[0], 0x4140), codes_f16x2(v[0], 0x4342),
                                                        codes_f16x2(v[1], 0x4140), codes_f16x2(v[1], 0x4342));
            *reinterpret_cast<uint4*>(dst + kChunkBytes) =
                make_uint4(codes_f16x2(v[2], 0x4140), codes_f16x2(v[2], 0x4342), codes_f16x2(v[3], 0x4140),
                           codes_f16x2(v[3], 0x4342));
        }
    };

    int t = blockIdx.x;
    TilePos p_cur{t / tiles_x, t % tiles_x};  // tiles t, t + G, t + 2 G
    TilePos p_next = advance(p_cur), p_next2 = advance(p_next);
    uint32_t e_cur = 0, e_next = 0, e_next2 = 0;  // their disparity entries
    if (t < tiles) {
        e_cur = load_entry(p_cur);
        if (warp == 1) load_box(p_cur);
        if (__syncthreads_or(!wait_bar(2))) failed = true;
        else build_a1(entry_winner(e_cur, a.disp_type));
    }
    if (t + (int)gridDim.x < tiles) e_next = load_entry(p_next);
    for (; t < tiles && !failed; t += gridDim.x) {
        const int y = p_cur.y, x0 = p_cur.tx * kM;
        // ---- conv1 biases into C1 (A1 was built while the previous tile's fc1 ran)
#pragma unroll
        for (int q = 0; q < 7; ++q) st32(tl + 32 * q, bias1);
        hand_to_issuer(true);
        // ---- conv1: window t = positions 3t .. 3t + 2 (N = 96; the last window N = 32)
        if (warp == 0) {  // MMA issue: whole warp, one elected lane
            fence_after();
            mma_ss(tm, dA1, dB1, kIdC1);
            mma_ss(tm + 96, dplus(dA1, 2 * kChunkBytes), dB1, kIdC1);
            mma_ss(tm + 192, dplus(dA1, 4 * kChunkBytes), dB1, kIdC1n);
            commit_to(0);
        }
        // the next tile's curve block (the box was last read by this tile's A1 build)
        if (warp == 1 && t + (int)gridDim.x < tiles) load_box(p_next);
        if (t + 2 * (int)gridDim.x < tiles) e_next2 = load_entry(p_next2);
        if (__syncthreads_or(!wait_bar(0))) { failed = true; break; }
        fence_after();
        // ---- conv1 epilogue: A2 position q (bf16) over the consumed C1 columns
#pragma unroll
        for (int q = 0; q < 6; q += 2) {
            float v[32], u[32];
            ld32x2(tl + 32 * q, tl + 32 * (q + 1), v, u);
            relu_bf16_to_tmem(tl + 16 * q, v);
            relu_bf16_to_tmem(tl + 16 * (q + 1), u);
        }
        {
            float v[32];
            ld32(tl + 32 * 6, v);
            relu_bf16_to_tmem(tl + 16 * 6, v);
        }
        bias_to_tmem(kC2, bias + 32);
        bias_to_tmem(kC2 + 32, bias + 32);
        hand_to_issuer(false);
        // ---- conv2 (A2 in TMEM): position r, taps j with input q = 3r + j - 1 in 0..6
        if (warp == 0) {  // MMA issue: whole warp, one elected lane
            fence_after();
#pragma unroll
            for (int r = 0; r < 2; ++r)
#pragma unroll
                for (int j = 0; j < 5; ++j) {
                    const int q = 3 * r + j - 1;
                    if (q < 0 || q >= 7) continue;
#pragma unroll
                    for (int h = 0; h < 2; ++h)
                        mma_ts(tm + kC2 + 32 * r, tm + 16 * q + 8 * h, dplus(dB2, (j * 4 + 2 * h) * 512), kIdC2);
                }
            commit_to(1);
        }
        if (__syncthreads_or(!wait_bar(1))) { failed = true; break; }
        fence_after();
        {
            float v[32], u[32];
            ld32x2(tl + kC2, tl + kC2 + 32, v, u);
            relu_bf16_to_tmem(tl + kA3, v);
            relu_bf16_to_tmem(tl + kA3 + 16, u);
        }
        bias_to_tmem(kC3, bias + 64);
        hand_to_issuer(false);
        // ---- conv3 (A3 in TMEM): taps 2, 3 on positions 0, 1
        if (warp == 0) {  // MMA issue: whole warp, one elected lane
            fence_after();
#pragma unroll
            for (int j = 0; j < 2; ++j)
#pragma unroll
                for (int h = 0; h < 2; ++h)
                    mma_ts(tm + kC3, tm + kA3 + 16 * j + 8 * h, dplus(dB3, (j * 4 + 2 * h) * 512), kIdC2);
            commit_to(0);
        }
        if (__syncthreads_or(!wait_bar(0))) { failed = true; break; }
        fence_after();
        {
            float v[32];
            ld32(tl + kC3, v);
            relu_bf16_to_tmem(tl + kA4, v);
        }
        bias_to_tmem(kC4, bias + 96);
        bias_to_tmem(kC4 + 32, bias + 128);
        hand_to_issuer(false);
        // ---- fc1 (A4 in TMEM): K = 32 (2 MMAs), N = 64
        if (warp == 0) {  // MMA issue: whole warp, one elected lane
            fence_after();
#pragma unroll
            for (int h = 0; h < 2; ++h) mma_ts(tm + kC4, tm + kA4 + 8 * h, dplus(dB4, 2 * h * 1024), kIdF1);
            commit_to(1);
        }
        // the next tile's A1 while fc1 runs (this tile's conv1 MMAs, the only
        // readers of A1, completed before the conv1 epilogue)
        bool box_ok = true;
        if (t + (int)gridDim.x < tiles) {
            box_ok = wait_bar(2);
            if (box_ok) build_a1(entry_winner(e_next, a.disp_type));
        }
        if (__syncthreads_or(!box_ok || !wait_bar(1))) { failed = true; break; }
        fence_after();
        // ---- fc1 epilogue + fc2
        {
            float v0[32], v1[32];
            ld32x2(tl + kC4, tl + kC4 + 32, v0, v1);
            float z[8] = {b5, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // eight independent chains
            const float4* w5v = reinterpret_cast<const float4*>(w5);  // 16-byte aligned in the image
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const float4 wa = w5v[c], wb = w5v[8 + c];
                z[0] = fmaf(wa.x, fmaxf(v0[4 * c], 0.f), z[0]);
                z[1] = fmaf(wa.y, fmaxf(v0[4 * c + 1], 0.f), z[1]);
                z[2] = fmaf(wa.z, fmaxf(v0[4 * c + 2], 0.f), z[2]);
                z[3] = fmaf(wa.w, fmaxf(v0[4 * c + 3], 0.f), z[3]);
                z[4] = fmaf(wb.x, fmaxf(v1[4 * c], 0.f), z[4]);
                z[5] = fmaf(wb.y, fmaxf(v1[4 * c + 1], 0.f), z[5]);
                z[6] = fmaf(wb.z, fmaxf(v1[4 * c + 2], 0.f), z[6]);
                z[7] = fmaf(wb.w, fmaxf(v1[4 * c + 3], 0.f), z[7]);
            }
            const float logit = ((z[0] + z[1]) + (z[2] + z[3])) + ((z[4] + z[5]) + (z[6] + z[7]));
            const float p = __fdividef(1.f, 1.f + __expf(-logit));  // 0 once exp overflows
            const int x = x0 + m;
            if (x < a.W) {
                if (a.score) reinterpret_cast<float*>(reinterpret_cast<char*>(a.score) + (size_t)y * a.score_pitch)[x] = p;
                if (a.checked) {  // same encoding as the cross-check's output map
                    char* crow = static_cast<char*>(a.checked) + (size_t)y * a.checked_pitch;
                    if (a.disp_type == CT_PIX_U8) {
                        reinterpret_cast<uint8_t*>(crow)[x] = p >= a.threshold ? uint8_t(e_cur) : uint8_t(0xFF);
                    } else {
                        const bool disp = e_cur >= CT_DISP_FIRST && e_cur <= CT_DISP_LAST;
                        reinterpret_cast<uint16_t*>(crow)[x] =
                            (disp && p < a.threshold) ? uint16_t(CT_DISP_INCONSISTENT) : uint16_t(e_cur);
                    }
                }
            }
        }
        e_cur = e_next;
        e_next = e_next2;
        p_cur = p_next;
        p_next = p_next2;
        p_next2 = advance(p_next2);
        fence_before();  // this tile's TMEM reads before the next tile's writes
    }
    // After a timeout, MMAs may still be in flight: wait (bounded) for every
    // commit not yet waited for before giving the TMEM back.
    if (failed && tid == 0) dev::report(a.status, CT_ETIMEOUT);
    if (failed && (tid & 31) == 0) {  // warp 0 issued the MMAs, warp 1 the TMA loads
        if (warp == 0) {
            for (uint32_t k = ph[0]; k < cm[0]; ++k) dev::mbar_wait_bounded(&bars[0], k & 1);
            for (uint32_t k = ph[1]; k < cm[1]; ++k) dev::mbar_wait_bounded(&bars[1], k & 1);
        } else if (warp == 1) {
            for (uint32_t k = ph[2]; k < cm[2]; ++k) dev::mbar_wait_bounded(&bars[2], k & 1);
        }
    }
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(kTmemCols) : "memory");
}

}  // namespace inf

// ---------------------------------------------------------------------------
// Training GEMMs on the tensor cores (tcgen05)
// ---------------------------------------------------------------------------
// The dense layers of training (conv2, conv3, fc1 forward; their data
// gradients; the weight gradients of conv2, conv3 and fc1) are GEMMs
//   D[M x N] (fp32, TMEM) = sum over passes of A_p[M x K] x B_p[N x K]^T
// with bf16 operands stored row-major (K contiguous) in global memory. conv1
// (one input channel, 1.1 K of the 14.5 K MAC per sample), the head and the
// elementwise steps stay on the CUDA cores.
namespace tg {

constexpr int kTM = 128;   // rows per tile = MMA M
constexpr int kKS = 64;    // K per pipeline stage: 8 panels of 8, 4 MMAs of K = 16
constexpr int kNT = 128;   // one warpgroup; warp w drains TMEM lanes 32 w .. 32 w + 31
constexpr int kMaxN = 256;

__host__ __device__ constexpr int stage_bytes(int N) { return (kTM + N) * kKS * 2; }
constexpr int kMaxSmem = 2 * stage_bytes(kMaxN) + 64;  // the largest launch (N = 256)

// Where a D element goes. kPlain: out[y * out_chunk + m * out_ld + n]. The
// weight-gradient layouts write into the parameter vector of chunk y
// (out = part, out_chunk = kParams): kW2T m = tap * 32 + in, n = out;
// kW3T m = (tap - 2) * 32 + in, n = out; kW4 m = hidden, n = in.
enum OutMap { kPlain = 0, kW2T = 1, kW3T = 2, kW4 = 3 };

struct GemmArgs {
    int N;           // columns of D: a multiple of 32, at most 256
    int npass;       // operand pairs accumulated into D (1 or 2)
    int klen;        // K of each pass
    int ksplit;      // K per blockIdx.y (a multiple of kKS)
    int m_valid;     // rows of D that are stored
    int map;         // OutMap
    float* out;
    size_t out_ld, out_chunk;
    uint32_t tmem_cols;  // power of two >= max(N, 32)
    int32_t* status;
};

// D (TMEM) = A x B (acc = 0) or D += A x B (acc = 1); whole warp, one elected lane issues
__device__ __forceinline__ void mma_ss_acc(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n.reg .pred p, e;\nsetp.ne.b32 p, %4, 0;\nelect.sync _|e, 0xffffffff;\n"
        "@e tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(id), "r"(acc)
        : "memory");
}

__device__ __forceinline__ int out_index(int map, int m, int n) {
    switch (map) {
        case kW2T: return m < 160 ? kOffW2 + n * 160 + (m % 32) * 5 + m / 32 : -1;
        case kW3T: return m < 64 ? kOffW3 + n * 160 + (m % 32) * 5 + 2 + m / 32 : -1;
        case kW4: return m < 64 ? kOffW4 + m * 32 + n : -1;
        default: return -1;
    }
}

// Operands through 3-D tensor maps over the row-major bf16 matrices: dims
// (8 elements, K / 8 panels, rows), one box per panel = 8 elements x rows, so
// that shared memory holds each 8-wide K panel as rows x 16 bytes: the
// canonical K-major layout without swizzle (core matrices of 8 rows x 16
// bytes, 128 bytes apart along M/N, one panel apart along K). Rows and K
// beyond the matrix read as 0.
__global__ void __launch_bounds__(kNT, 1) gemm_kernel(const __grid_constant__ CUtensorMap a0,
                                                     const __grid_constant__ CUtensorMap b0,
                                                     const __grid_constant__ CUtensorMap a1,
                                                     const __grid_constant__ CUtensorMap b1, GemmArgs g) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int SB = stage_bytes(g.N);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * SB);  // full[2], free[2], done
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 5);
    const int m0 = blockIdx.x * kTM;
    const int k0 = blockIdx.y * g.ksplit;
    const int kend = min(k0 + g.ksplit, g.klen);
    const int nk = kend > k0 ? (kend - k0 + kKS - 1) / kKS : 0;  // stages per pass
    const int total = nk * g.npass;
    if (tid == 0) {
        for (int i = 0; i < 5; ++i) dev::mbar_init(&bars[i], 1);
        dev::fence_barrier_init();
        dev::prefetch_tmap(&a0);
        dev::prefetch_tmap(&b0);
        if (g.npass > 1) {
            dev::prefetch_tmap(&a1);
            dev::prefetch_tmap(&b1);
        }
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dev::smem_u32(tslot)),
                     "r"(g.tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    inf::fence_before();
    __syncthreads();
    inf::fence_after();
    const uint32_t tm = *tslot;
    // instruction descriptor: bf16 x bf16 -> fp32, both K-major, M = 128
    const uint32_t id = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(g.N >> 3) << 17) | (uint32_t(kTM >> 4) << 24);

    // warp 0: lane 0 loads stages, the whole warp issues the MMAs
    bool ok = true;
    int loaded = 0, consumed = 0;  // stages loaded / consumed (warp 0)
    if (warp == 0) {
        auto load = [&](int it) {
            if (lane == 0) {
                const int s = it & 1, pass = it / nk, kk = k0 + (it % nk) * kKS;
                const CUtensorMap* ma = pass ? &a1 : &a0;
                const CUtensorMap* mb = pass ? &b1 : &b0;
                unsigned char* sa = smem + s * SB;
                unsigned char* sb = sa + kTM * kKS * 2;
                dev::mbar_arrive_expect_tx(&bars[s], uint32_t(SB));
#pragma unroll
                for (int c = 0; c < kKS / 8; ++c) {
                    dev::tma_load_3d(sa + c * kTM * 16, ma, 0, kk / 8 + c, m0, &bars[s]);
                    dev::tma_load_3d(sb + c * g.N * 16, mb, 0, kk / 8 + c, 0, &bars[s]);
                }
            }
            __syncwarp();
        };
        uint32_t ph_full = 0u, ph_free = 0u;  // phase bit s of stage s's barriers
        for (; loaded < total && loaded < 2; ++loaded) load(loaded);
        for (int it = 0; it < total && ok; ++it) {
            const int s = it & 1;
            ok = __all_sync(0xffffffffu, dev::mbar_wait_bounded(&bars[s], (ph_full >> s) & 1u));
            if (!ok) break;
            ph_full ^= 1u << s;
            ++consumed;
            inf::fence_after();
            const uint32_t sa = dev::smem_u32(smem + s * SB), sb = sa + kTM * kKS * 2;
#pragma unroll
            for (int q = 0; q < kKS / 16; ++q)
                mma_ss_acc(tm, inf::sdesc(sa + q * 2 * kTM * 16, kTM * 16), inf::sdesc(sb + q * 2 * g.N * 16, g.N * 16),
                           id, (it > 0 || q > 0) ? 1u : 0u);
            inf::commit(&bars[2 + s]);  // stage s is free once these MMAs complete
            if (it + 2 < total) {
                ok = __all_sync(0xffffffffu, dev::mbar_wait_bounded(&bars[2 + s], (ph_free >> s) & 1u));
                if (!ok) break;
                ph_free ^= 1u << s;
                load(it + 2);
                ++loaded;
            }
        }
        inf::commit(&bars[4]);  // every MMA issued so far
    }
    // all threads: the accumulator is complete (or the loop gave up)
    const bool done = dev::mbar_wait_bounded(&bars[4], 0);
    const bool fail = __syncthreads_or(!ok || !done);
    inf::fence_after();
    if (fail) {
        if (tid == 0) dev::report(g.status, CT_ETIMEOUT);
        // wait (bounded) for the stage loads still in flight before leaving
        if (warp == 0 && lane == 0)
            for (int it = consumed; it < loaded; ++it) dev::mbar_wait_bounded(&bars[it & 1], ((it >> 1) & 1));
    } else if (total > 0) {
        const int row = m0 + tid;
        const uint32_t tl = tm + (uint32_t(warp * 32) << 16);
        float* outc = g.out + (size_t)blockIdx.y * g.out_chunk;
        for (int c0 = 0; c0 < g.N; c0 += 32) {
            float v[32];
            inf::ld32(tl + c0, v);
            if (row < g.m_valid) {
                if (g.map == kPlain) {
                    float* o = outc + (size_t)row * g.out_ld + c0;
#pragma unroll
                    for (int j = 0; j < 32; j += 4) *reinterpret_cast<float4*>(o + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
                } else {
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        const int p = out_index(g.map, row, c0 + j);
                        if (p >= 0) outc[p] = v[j];
                    }
                }
            }
        }
    }
    inf::fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(g.tmem_cols) : "memory");
}

// The bf16 B operands of the training GEMMs from the working weights wq:
//   w2f [32 out][160 = tap * 32 + in]      conv2 forward
//   w3f [32 out][64 = (tap - 2) * 32 + in]  conv3 forward (taps 2, 3)
//   w4f [64 hidden][32 in]                  fc1 forward
//   w4t [32 in][64 hidden]                  fc1 data gradient
//   w3t [64 = (tap - 2) * 32 + in][32 out]  conv3 data gradient
//   w2t [224 = q * 32 + in][64 = r * 32 + out] conv2 data gradient: W2[out][in][q - 3 r + 1] (0 outside the taps)
struct TrainW {
    uint16_t *w2f, *w3f, *w4f, *w4t, *w3t, *w2t;
};
constexpr int kTrainWElems = 32 * 160 + 32 * 64 + 64 * 32 + 32 * 64 + 64 * 32 + 224 * 64;

__global__ void pack_train_weights_kernel(const float* wq, TrainW w) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < kTrainWElems; k += gridDim.x * blockDim.x) {
        int e = k;
        if (e < 32 * 160) {
            const int o = e / 160, t = (e % 160) / 32, i = e % 32;
            w.w2f[e] = bf16_bits(wq[kOffW2 + o * 160 + i * 5 + t]);
            continue;
        }
        e -= 32 * 160;
        if (e < 32 * 64) {
            const int o = e / 64, t = (e % 64) / 32, i = e % 32;
            w.w3f[e] = bf16_bits(wq[kOffW3 + o * 160 + i * 5 + 2 + t]);
            continue;
        }
        e -= 32 * 64;
        if (e < 64 * 32) {
            w.w4f[e] = bf16_bits(wq[kOffW4 + e]);
            continue;
        }
        e -= 64 * 32;
        if (e < 32 * 64) {
            const int i = e / 64, hh = e % 64;
            w.w4t[e] = bf16_bits(wq[kOffW4 + hh * 32 + i]);
            continue;
        }
        e -= 32 * 64;
        if (e < 64 * 32) {
            const int t = e / (32 * 32), i = (e / 32) % 32, o = e % 32;
            w.w3t[e] = bf16_bits(wq[kOffW3 + o * 160 + i * 5 + 2 + t]);
            continue;
        }
        e -= 64 * 32;
        {
            const int q = e / (32 * 64), i = (e / 64) % 32, r = (e % 64) / 32, o = e % 32;
            const int j = q - 3 * r + 1;
            w.w2t[e] = (j >= 0 && j < 5) ? bf16_bits(wq[kOffW2 + o * 160 + i * 5 + j]) : uint16_t(0);
        }
    }
}

}  // namespace tg

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
uint16_t f32_to_bf16_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    if ((u & 0x7FFFFFFFu) > 0x7F800000u) return uint16_t((u >> 16) | 0x40);  // NaN
    u += 0x7FFFu + ((u >> 16) & 1u);
    return uint16_t(u >> 16);
}
float bf16_bits_to_f32(uint16_t b) {
    const uint32_t u = uint32_t(b) << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
// Exact conversion of a bf16 value to f16 bits; returns false if the value
// is not representable in f16 (outside its range or below its precision).
bool bf16_to_f16_exact(float v, uint16_t* out) {
    const __half h = __float2half_rn(v);
    *out = __half_as_ushort(h);
    return __half2float(h) == v;
}

struct ConfNetHandle : ct_handle {
    ConfNetHandle() : ct_handle(Kind::ConfNet) {}
    ~ConfNetHandle() override {
        if (device >= 0) cudaSetDevice(device);
        cudaFree(arena);
    }
    int max_batch = 0;
    unsigned char* arena = nullptr;
    float *master = nullptr, *m = nullptr, *v = nullptr, *wq = nullptr, *grad = nullptr, *part = nullptr;
    float* loss_out = nullptr;
    unsigned char* wimg = nullptr;  // packed inference weights
    tg::TrainW tw{};                // bf16 B operands of the training GEMMs
    Act act{};
    int steps = 0;
    bool wimg_dirty = true;
    int sms = 148;
};

ConfNetHandle* as_net(ct_handle* h) {
    return (h && h->kind == Kind::ConfNet) ? static_cast<ConfNetHandle*>(h) : nullptr;
}

int chunks_for(int n) { return (n + kChunk - 1) / kChunk; }

// A row-major bf16 matrix [rows][K] (pitch in elements) as a GEMM operand
// map: dims (8, K / 8, rows), one 8-wide panel x box_rows rows per box.
int operand_map(CUtensorMap* m, const uint16_t* base, int rows, int K, size_t pitch, int box_rows) {
    const uint64_t dims[3] = {8, uint64_t((K + 7) / 8), uint64_t(rows)};
    const uint64_t strides[2] = {16, pitch * 2};
    const uint32_t box[3] = {8, 1, uint32_t(box_rows)};
    return make_tmap_nd(m, base, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, 3, dims, strides, box);
}

// D = sum over passes of A_p x B_p^T on the tensor cores (tg::gemm_kernel):
// M rows of A, N rows of B (a multiple of 32), K = klen split into ksplit
// per blockIdx.y.
int tc_gemm(ConfNetHandle* h, const CUtensorMap& a0, const CUtensorMap& b0, const CUtensorMap* a1,
            const CUtensorMap* b1, int M, int N, int klen, int ksplit, int map, float* out, size_t out_ld,
            size_t out_chunk, cudaStream_t s) {
    tg::GemmArgs g{};
    g.N = N;
    g.npass = a1 ? 2 : 1;
    g.klen = klen;
    g.ksplit = ksplit;
    g.m_valid = M;
    g.map = map;
    g.out = out;
    g.out_ld = out_ld;
    g.out_chunk = out_chunk;
    g.tmem_cols = N <= 32 ? 32u : N <= 64 ? 64u : N <= 128 ? 128u : 256u;
    g.status = h->d_status;
    const dim3 grid((M + tg::kTM - 1) / tg::kTM, (klen + ksplit - 1) / ksplit);
    tg::gemm_kernel<<<grid, tg::kNT, 2 * tg::stage_bytes(N) + 64, s>>>(a0, b0, a1 ? *a1 : a0, b1 ? *b1 : b0, g);
    CT_LAUNCH_CHECK();
    return CT_OK;
}

// forward (+ backward when labels are given) of n samples on stream s:
// conv1, the head and the elementwise steps on the CUDA cores, the dense
// layers (conv2, conv3, fc1), their data gradients and their weight
// gradients as bf16 GEMMs with fp32 accumulation on the tensor cores
int run_train_graph(ConfNetHandle* h, const uint8_t* x, const uint8_t* labels, int n, float* scores,
                    cudaStream_t s) {
    const Act& A = h->act;
    const dim3 b32(32, kSY), b64(64, 8), be(32, 8);
    const int g32 = (n + kSY - 1) / kSY, g64 = (n + 7) / 8, ge = (n + 7) / 8;
    const int n8 = (n + 7) & ~7;
    const size_t lt = size_t(A.ldt);
    tg::pack_train_weights_kernel<<<(tg::kTrainWElems + 255) / 256, 256, 0, s>>>(h->wq, h->tw);
    fwd1_kernel<<<g32, b32, 0, s>>>(x, h->wq, A, n);
    CT_LAUNCH_CHECK();
    const int kS = tg::kKS;
    auto ks = [&](int k) { return (k + kS - 1) / kS * kS; };  // whole K in one CTA
    CUtensorMap ma, mb, ma2, mb2;
    // conv2: position r reads slots 3 r .. 3 r + 4 of a1p (160 contiguous values)
    if (int rc = operand_map(&mb, h->tw.w2f, 32, 160, 160, 32)) return rc;
    for (int r = 0; r < kR; ++r) {
        if (int rc = operand_map(&ma, A.a1p + 96 * r, n, 160, 256, tg::kTM)) return rc;
        if (int rc = tc_gemm(h, ma, mb, nullptr, nullptr, n, 32, 160, ks(160), tg::kPlain, A.d + 32 * r, 64, 0, s))
            return rc;
    }
    ep_fwd_kernel<<<ge, be, 0, s>>>(A.d, 64, h->wq + kOffB2, 32, 1, A.a2, A.a2b, A.a2t, A.ldt, n);
    // conv3 (taps 2, 3 over both positions) and fc1
    if (int rc = operand_map(&ma, A.a2b, n, 64, 64, tg::kTM)) return rc;
    if (int rc = operand_map(&mb, h->tw.w3f, 32, 64, 64, 32)) return rc;
    if (int rc = tc_gemm(h, ma, mb, nullptr, nullptr, n, 32, 64, ks(64), tg::kPlain, A.d, 32, 0, s)) return rc;
    ep_fwd_kernel<<<ge, be, 0, s>>>(A.d, 32, h->wq + kOffB3, 32, 1, A.a3, A.a3b, A.a3t, A.ldt, n);
    if (int rc = operand_map(&ma, A.a3b, n, 32, 32, tg::kTM)) return rc;
    if (int rc = operand_map(&mb, h->tw.w4f, 64, 32, 32, 64)) return rc;
    if (int rc = tc_gemm(h, ma, mb, nullptr, nullptr, n, 64, 32, ks(32), tg::kPlain, A.d, 64, 0, s)) return rc;
    ep_fwd_kernel<<<ge, be, 0, s>>>(A.d, 64, h->wq + kOffB4, 64, 0, A.a4, nullptr, nullptr, A.ldt, n);
    head_kernel<<<(n + 255) / 256, 256, 0, s>>>(h->wq, A, labels, 1.f / float(n), scores, n);
    CT_LAUNCH_CHECK();
    if (!labels) return CT_OK;
    // data gradients
    bwd4_kernel<<<g64, b64, 0, s>>>(h->wq, A, n);
    if (int rc = operand_map(&ma, A.dz4b, n, 64, 64, tg::kTM)) return rc;
    if (int rc = operand_map(&mb, h->tw.w4t, 32, 64, 64, 32)) return rc;
    if (int rc = tc_gemm(h, ma, mb, nullptr, nullptr, n, 32, 64, ks(64), tg::kPlain, A.d, 32, 0, s)) return rc;
    ep_bwd_kernel<<<ge, be, 0, s>>>(A.d, 32, A.a3, A.dz3, A.dz3b, A.dz3t, A.ldt, n);
    if (int rc = operand_map(&ma, A.dz3b, n, 32, 32, tg::kTM)) return rc;
    if (int rc = operand_map(&mb, h->tw.w3t, 64, 32, 32, 64)) return rc;
    if (int rc = tc_gemm(h, ma, mb, nullptr, nullptr, n, 64, 32, ks(32), tg::kPlain, A.d, 64, 0, s)) return rc;
    ep_bwd_kernel<<<ge, be, 0, s>>>(A.d, 64, A.a2, A.dz2, A.dz2b, A.dz2t, A.ldt, n);
    if (int rc = operand_map(&ma, A.dz2b, n, 64, 64, tg::kTM)) return rc;
    if (int rc = operand_map(&mb, h->tw.w2t, 224, 64, 64, 224)) return rc;
    if (int rc = tc_gemm(h, ma, mb, nullptr, nullptr, n, 224, 64, ks(64), tg::kPlain, A.d, 224, 0, s)) return rc;
    ep_bwd_kernel<<<ge, be, 0, s>>>(A.d, 224, A.a1, A.dm1, nullptr, nullptr, A.ldt, n);
    // weight gradients per chunk of kChunk samples into part[chunk][param]
    // conv2: sum over positions r of a1p slots 3 r .. 3 r + 4 (rows) x dz2 position r
    if (int rc = operand_map(&ma, A.a1pt, 160, n8, lt, tg::kTM)) return rc;
    if (int rc = operand_map(&mb, A.dz2t, 32, n8, lt, 32)) return rc;
    if (int rc = operand_map(&ma2, A.a1pt + 96 * lt, 160, n8, lt, tg::kTM)) return rc;
    if (int rc = operand_map(&mb2, A.dz2t + 32 * lt, 32, n8, lt, 32)) return rc;
    if (int rc = tc_gemm(h, ma, mb, &ma2, &mb2, 160, 32, n8, kChunk, tg::kW2T, h->part, 0, kParams, s)) return rc;
    if (int rc = operand_map(&ma, A.a2t, 64, n8, lt, tg::kTM)) return rc;
    if (int rc = operand_map(&mb, A.dz3t, 32, n8, lt, 32)) return rc;
    if (int rc = tc_gemm(h, ma, mb, nullptr, nullptr, 64, 32, n8, kChunk, tg::kW3T, h->part, 0, kParams, s)) return rc;
    if (int rc = operand_map(&ma, A.dz4t, 64, n8, lt, tg::kTM)) return rc;
    if (int rc = operand_map(&mb, A.a3t, 32, n8, lt, 32)) return rc;
    if (int rc = tc_gemm(h, ma, mb, nullptr, nullptr, 64, 32, n8, kChunk, tg::kW4, h->part, 0, kParams, s)) return rc;
    wgrad_kernel<<<dim3(chunks_for(n), 5), 256, 0, s>>>(x, A, n, h->part);
    CT_LAUNCH_CHECK();
    return CT_OK;
}

// Packs master weights into the inference image (host side).
int pack_weights(ConfNetHandle* h) {
    using namespace inf;
    std::vector<float> p(kParams);
    CT_CUDA_TRY(cudaMemcpy(p.data(), h->master, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
    std::vector<unsigned char> img(kWBytes, 0);
    auto put16 = [&](int off, uint16_t v) { std::memcpy(&img[off], &v, 2); };
    auto bf = [&](int idx) { return bf16_bits_to_f32(f32_to_bf16_bits(p[idx])); };
    // B1: rows = pp * 32 + channel (pp = position in a conv1 window), tap j
    // of position pp at K = 5 pp + j (K = 15 is zero); 2 chunks of 96 rows
    for (int pp = 0; pp < 3; ++pp)
        for (int ch = 0; ch < 32; ++ch)
            for (int j = 0; j < 5; ++j) {
                const int k = 5 * pp + j, n = pp * 32 + ch;
                uint16_t hb;
                if (!bf16_to_f16_exact(bf(kOffW1 + ch * 5 + j), &hb))
                    return fail(CT_EINVAL, "conv1 weight %d (%g) is not exact in f16", ch * 5 + j,
                                double(bf(kOffW1 + ch * 5 + j)));
                put16(kB1 + (k / 8) * 1536 + n * 16 + (k % 8) * 2, hb);
            }
    // B2: rows o, K = tap * 32 + in; B3: rows o, K = (tap - 2) * 32 + in, taps 2, 3
    for (int o = 0; o < 32; ++o)
        for (int i = 0; i < 32; ++i) {
            for (int j = 0; j < 5; ++j) {
                const int k = j * 32 + i;
                put16(kB2 + (k / 8) * 512 + o * 16 + (k % 8) * 2, f32_to_bf16_bits(p[kOffW2 + o * 160 + i * 5 + j]));
            }
            for (int j = 2; j < 4; ++j) {
                const int k = (j - 2) * 32 + i;
                put16(kB3 + (k / 8) * 512 + o * 16 + (k % 8) * 2, f32_to_bf16_bits(p[kOffW3 + o * 160 + i * 5 + j]));
            }
        }
    // B4: rows h, K = in
    for (int hh = 0; hh < 64; ++hh)
        for (int i = 0; i < 32; ++i)
            put16(kB4 + (i / 8) * 1024 + hh * 16 + (i % 8) * 2, f32_to_bf16_bits(p[kOffW4 + hh * 32 + i]));
    float* bias = reinterpret_cast<float*>(&img[kBias]);
    for (int k = 0; k < 32; ++k) bias[k] = p[kOffB1 + k];
    for (int k = 0; k < 32; ++k) bias[32 + k] = p[kOffB2 + k];
    for (int k = 0; k < 32; ++k) bias[64 + k] = p[kOffB3 + k];
    for (int k = 0; k < 64; ++k) bias[96 + k] = p[kOffB4 + k];
    for (int k = 0; k < 64; ++k) bias[160 + k] = bf(kOffW5 + k);
    bias[224] = p[kOffB5];
    CT_CUDA_TRY(cudaMemcpy(h->wimg, img.data(), kWBytes, cudaMemcpyHostToDevice));
    h->wimg_dirty = false;
    return CT_OK;
}

int upload_params(ConfNetHandle* h, const float* host) {
    std::vector<float> q(host, host + kParams);
    for (int p = 0; p < kParams; ++p)
        if (is_weight(p)) q[p] = bf16_bits_to_f32(f32_to_bf16_bits(q[p]));
    CT_CUDA_TRY(cudaMemcpy(h->master, host, sizeof(float) * kParams, cudaMemcpyHostToDevice));
    CT_CUDA_TRY(cudaMemcpy(h->wq, q.data(), sizeof(float) * kParams, cudaMemcpyHostToDevice));
    CT_CUDA_TRY(cudaMemset(h->m, 0, sizeof(float) * kParams));
    CT_CUDA_TRY(cudaMemset(h->v, 0, sizeof(float) * kParams));
    h->steps = 0;
    h->wimg_dirty = true;
    return CT_OK;
}

}  // namespace cn
}  // namespace ct

using namespace ct;
using namespace ct::cn;

extern "C" {

int ct_confnet_create(ct_handle** out) {
    clear_error();
    if (!out) return fail(CT_EINVAL, "null output handle pointer");
    *out = new ConfNetHandle();
    return CT_OK;
}

int ct_confnet_configure(ct_handle* hh, int32_t device, int32_t max_batch) {
    clear_error();
    auto* h = as_net(hh);
    if (!h) return fail(CT_ESTATE, "not a confidence-net handle");
    if (max_batch < 1 || max_batch > (1 << 22)) return fail(CT_EINVAL, "max_batch must be 1..4194304");
    if (int rc = use_device(device)) return rc;
    h->device = device;
    if (int rc = h->init_status()) return rc;
    CT_CUDA_TRY(cudaFuncSetAttribute(inf::infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, inf::kSmem));
    CT_CUDA_TRY(cudaFuncSetAttribute(tg::gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tg::kMaxSmem));
    h->sms = sm_count(device);
    const size_t n = size_t(max_batch);
    size_t bytes = 0;
    auto take = [&](size_t b) { const size_t o = bytes; bytes += (b + 255) / 256 * 256; return o; };
    const size_t o_master = take(4 * kParams), o_m = take(4 * kParams), o_v = take(4 * kParams),
                 o_wq = take(4 * kParams), o_grad = take(4 * kParams),
                 o_part = take(4 * size_t(kParams) * chunks_for(max_batch)), o_loss = take(16),
                 o_wimg = take(inf::kWBytes), o_a1 = take(4 * 224 * n), o_a2 = take(4 * 64 * n),
                 o_a3 = take(4 * 32 * n), o_a4 = take(4 * 64 * n), o_logit = take(4 * n), o_dl = take(4 * n),
                 o_ls = take(4 * n), o_dz4 = take(4 * 64 * n), o_dz3 = take(4 * 32 * n), o_dz2 = take(4 * 64 * n),
                 o_dm1 = take(4 * 224 * n);
    const size_t ldt = (n + 7) / 8 * 8;  // transposed operands: samples per row, a multiple of 8
    const size_t o_a1p = take(2 * 256 * n), o_a1pt = take(2 * 256 * ldt), o_a2b = take(2 * 64 * n),
                 o_a2t = take(2 * 64 * ldt), o_a3b = take(2 * 32 * n), o_a3t = take(2 * 32 * ldt),
                 o_dz4b = take(2 * 64 * n), o_dz4t = take(2 * 64 * ldt), o_dz3b = take(2 * 32 * n),
                 o_dz3t = take(2 * 32 * ldt), o_dz2b = take(2 * 64 * n), o_dz2t = take(2 * 64 * ldt),
                 o_d = take(4 * 224 * n), o_tw = take(2 * tg::kTrainWElems);
    cudaFree(h->arena);
    h->arena = nullptr;
    if (cudaMalloc(&h->arena, bytes) != cudaSuccess) return fail(CT_ENOMEM, "confidence-net scratch (%zu bytes)", bytes);
    CT_CUDA_TRY(cudaMemset(h->arena, 0, bytes));
    unsigned char* A = h->arena;
    h->master = reinterpret_cast<float*>(A + o_master);
    h->m = reinterpret_cast<float*>(A + o_m);
    h->v = reinterpret_cast<float*>(A + o_v);
    h->wq = reinterpret_cast<float*>(A + o_wq);
    h->grad = reinterpret_cast<float*>(A + o_grad);
    h->part = reinterpret_cast<float*>(A + o_part);
    h->loss_out = reinterpret_cast<float*>(A + o_loss);
    h->wimg = A + o_wimg;
    h->act.a1 = reinterpret_cast<float*>(A + o_a1);
    h->act.a2 = reinterpret_cast<float*>(A + o_a2);
    h->act.a3 = reinterpret_cast<float*>(A + o_a3);
    h->act.a4 = reinterpret_cast<float*>(A + o_a4);
    h->act.logit = reinterpret_cast<float*>(A + o_logit);
    h->act.dl = reinterpret_cast<float*>(A + o_dl);
    h->act.loss = reinterpret_cast<float*>(A + o_ls);
    h->act.dz4 = reinterpret_cast<float*>(A + o_dz4);
    h->act.dz3 = reinterpret_cast<float*>(A + o_dz3);
    h->act.dz2 = reinterpret_cast<float*>(A + o_dz2);
    h->act.dm1 = reinterpret_cast<float*>(A + o_dm1);
    auto u16 = [&](size_t o) { return reinterpret_cast<uint16_t*>(A + o); };
    h->act.a1p = u16(o_a1p);
    h->act.a1pt = u16(o_a1pt);
    h->act.a2b = u16(o_a2b);
    h->act.a2t = u16(o_a2t);
    h->act.a3b = u16(o_a3b);
    h->act.a3t = u16(o_a3t);
    h->act.dz4b = u16(o_dz4b);
    h->act.dz4t = u16(o_dz4t);
    h->act.dz3b = u16(o_dz3b);
    h->act.dz3t = u16(o_dz3t);
    h->act.dz2b = u16(o_dz2b);
    h->act.dz2t = u16(o_dz2t);
    h->act.d = reinterpret_cast<float*>(A + o_d);
    h->act.ldt = int(ldt);
    uint16_t* tw = u16(o_tw);
    h->tw.w2f = tw;
    h->tw.w3f = h->tw.w2f + 32 * 160;
    h->tw.w4f = h->tw.w3f + 32 * 64;
    h->tw.w4t = h->tw.w4f + 64 * 32;
    h->tw.w3t = h->tw.w4t + 32 * 64;
    h->tw.w2t = h->tw.w3t + 64 * 32;
    h->max_batch = max_batch;
    h->configured = true;
    return ct_confnet_init(hh, 1);
}

int ct_confnet_init(ct_handle* hh, uint64_t seed) {
    clear_error();
    auto* h = as_net(hh);
    if (!h || !h->configured) return fail(CT_ESTATE, "not a configured confidence-net handle");
    if (int rc = use_device(h->device)) return rc;
    // SplitMix64 + Box-Muller, He-style scales (conv1 scaled for inputs 0..255)
    uint64_t st = seed * 0x9E3779B97F4A7C15ull + 0x2545F4914F6CDD1Dull;
    auto u01 = [&]() {
        st += 0x9E3779B97F4A7C15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double(z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    };
    auto normal = [&]() { return std::sqrt(-2.0 * std::log(u01())) * std::cos(6.283185307179586 * u01()); };
    std::vector<float> p(kParams, 0.f);
    auto fill = [&](int off, int count, double sd) {
        for (int k = 0; k < count; ++k) p[off + k] = float(sd * normal());
    };
    fill(kOffW1, 160, 1.0 / (std::sqrt(5.0) * 128.0));
    fill(kOffW2, 5120, std::sqrt(2.0 / 160));
    fill(kOffW3, 5120, std::sqrt(2.0 / 128));
    fill(kOffW4, 2048, std::sqrt(2.0 / 32));
    fill(kOffW5, 64, std::sqrt(1.0 / 64));
    return upload_params(h, p.data());
}

int ct_confnet_set_params(ct_handle* hh, const float* params, int32_t n) {
    clear_error();
    auto* h = as_net(hh);
    if (!h || !h->configured) return fail(CT_ESTATE, "not a configured confidence-net handle");
    if (!params || n != kParams) return fail(CT_EINVAL, "need %d parameters", kParams);
    if (int rc = use_device(h->device)) return rc;
    return upload_params(h, params);
}

int ct_confnet_get_params(ct_handle* hh, float* params, int32_t n) {
    clear_error();
    auto* h = as_net(hh);
    if (!h || !h->configured) return fail(CT_ESTATE, "not a configured confidence-net handle");
    if (!params || n != kParams) return fail(CT_EINVAL, "need %d parameters", kParams);
    if (int rc = use_device(h->device)) return rc;
    CT_CUDA_TRY(cudaDeviceSynchronize());
    CT_CUDA_TRY(cudaMemcpy(params, h->master, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
    return CT_OK;
}

// The disparity map must match the curve volume's size; U8 or U16 encoding.
static int check_disp_for(const ct_image* disp, const ct_curves* curves) {
    if (int rc = check_image(disp, "disp", (1u << CT_PIX_U8) | (1u << CT_PIX_U16))) return rc;
    if (disp->width != curves->width || disp->height != curves->height)
        return fail(CT_EFORMAT, "disparity map and curve volume differ in size");
    return CT_OK;
}

int ct_confnet_gather(ct_handle* hh, uint8_t* samples, const ct_curves* curves, const ct_image* disp,
                      const int32_t* xy, int32_t n, ct_stream stream) {
    clear_error();
    auto* h = as_net(hh);
    if (!h || !h->configured) return fail(CT_ESTATE, "not a configured confidence-net handle");
    if (!samples || !curves || !curves->ptr || !xy || n < 0) return fail(CT_EINVAL, "null argument");
    if (curves->disp_count != kLen) return fail(CT_EFORMAT, "the confidence net reads curves of 128 disparities");
    if (int rc = check_disp_for(disp, curves)) return rc;
    if (n == 0) return CT_OK;
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    gather_kernel<<<(n + 7) / 8, 256, 0, s>>>(samples, static_cast<const uint32_t*>(curves->ptr),
                                              curves->pitch_bytes / 4, curves->width, curves->height, disp->ptr,
                                              disp->pitch_bytes, disp->type, xy, n, h->d_status);
    CT_LAUNCH_CHECK();
    return CT_OK;
}

int ct_confnet_loss_grad(ct_handle* hh, const uint8_t* samples, const uint8_t* labels, int32_t n, float* grad,
                         float* loss, ct_stream stream) {
    clear_error();
    auto* h = as_net(hh);
    if (!h || !h->configured) return fail(CT_ESTATE, "not a configured confidence-net handle");
    if (!samples || !labels || n < 1 || n > h->max_batch) return fail(CT_EINVAL, "bad samples/labels or n");
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    if (int rc = run_train_graph(h, samples, labels, n, nullptr, s)) return rc;
    reduce_adam_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(h->part, chunks_for(n), grad ? grad : h->grad, h->master,
                                                            h->m, h->v, h->wq, AdamArgs{0, 0, 0, 0, 0, 1, 1});
    if (loss) loss_mean_kernel<<<1, 256, 0, s>>>(h->act.loss, n, loss);
    CT_LAUNCH_CHECK();
    return CT_OK;
}

int ct_confnet_train_step(ct_handle* hh, const uint8_t* samples, const uint8_t* labels, int32_t n, float lr,
                          float* loss, ct_stream stream) {
    clear_error();
    auto* h = as_net(hh);
    if (!h || !h->configured) return fail(CT_ESTATE, "not a configured confidence-net handle");
    if (!samples || !labels || n < 1 || n > h->max_batch) return fail(CT_EINVAL, "bad samples/labels or n");
    if (!(lr > 0.f)) return fail(CT_EINVAL, "lr must be > 0");
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    if (int rc = run_train_graph(h, samples, labels, n, nullptr, s)) return rc;
    ++h->steps;
    const float b1 = 0.9f, b2 = 0.999f;
    AdamArgs aa{1, lr, b1, b2, 1e-8f, float(1.0 - std::pow(double(b1), h->steps)),
                float(1.0 - std::pow(double(b2), h->steps))};
    reduce_adam_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(h->part, chunks_for(n), h->grad, h->master, h->m, h->v,
                                                            h->wq, aa);
    if (loss) loss_mean_kernel<<<1, 256, 0, s>>>(h->act.loss, n, loss);
    CT_LAUNCH_CHECK();
    h->wimg_dirty = true;
    return CT_OK;
}

int ct_confnet_scores(ct_handle* hh, float* scores, const uint8_t* samples, int32_t n, ct_stream stream) {
    clear_error();
    auto* h = as_net(hh);
    if (!h || !h->configured) return fail(CT_ESTATE, "not a configured confidence-net handle");
    if (!scores || !samples || n < 1 || n > h->max_batch) return fail(CT_EINVAL, "bad arguments");
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    return run_train_graph(h, samples, nullptr, n, scores, s);
}

int ct_confnet_infer(ct_handle* hh, const ct_image* score, const ct_curves* curves, const ct_image* disp,
                     const ct_image* checked, float threshold, ct_stream stream) {
    clear_error();
    auto* h = as_net(hh);
    if (!h || !h->configured) return fail(CT_ESTATE, "not a configured confidence-net handle");
    if (!score && !checked) return fail(CT_EINVAL, "no output requested");
    if (!curves || !curves->ptr) return fail(CT_EINVAL, "null curve volume");
    if (curves->disp_count != kLen) return fail(CT_EFORMAT, "the confidence net reads curves of 128 disparities");
    if (int rc = check_disp_for(disp, curves)) return rc;
    if (score) {
        if (int rc = check_image(score, "score", 1u << CT_PIX_F32)) return rc;
        if (curves->width != score->width || curves->height != score->height)
            return fail(CT_EFORMAT, "score map and curve volume differ in size");
    }
    if (checked) {
        if (int rc = check_image(checked, "checked", 1u << disp->type)) return rc;
        if (checked->width != disp->width || checked->height != disp->height)
            return fail(CT_EFORMAT, "checked map and disparity map differ in size");
    }
    if (reinterpret_cast<uintptr_t>(curves->ptr) % 16 || curves->pitch_bytes % 16 ||
        curves->pitch_bytes < 4 * (size_t(curves->width) + 2))
        return fail(CT_EINVAL, "curve volume needs a 16-byte aligned pointer and pitch >= 4 * (width + 2)");
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (h->wimg_dirty) {
        if (h->last_stream) CT_CUDA_TRY(cudaStreamSynchronize(h->last_stream));
        if (int rc = pack_weights(h)) return rc;
    }
    h->last_stream = s;
    inf::InferArgs a{};
    a.curve = static_cast<const uint32_t*>(curves->ptr);
    a.curve_pitch = curves->pitch_bytes / 4;
    a.groups = kLen / 4;
    a.disp = disp->ptr;
    a.disp_pitch = disp->pitch_bytes;
    a.disp_type = disp->type;
    a.W = curves->width;
    a.H = curves->height;
    a.score = score ? static_cast<float*>(score->ptr) : nullptr;
    a.score_pitch = score ? score->pitch_bytes : 0;
    a.checked = checked ? checked->ptr : nullptr;
    a.checked_pitch = checked ? checked->pitch_bytes : 0;
    a.threshold = threshold;
    a.wimg = reinterpret_cast<const uint4*>(h->wimg);
    a.status = h->d_status;
    const int tiles = ((a.W + inf::kM - 1) / inf::kM) * a.H;
    const int grid = tiles < 2 * h->sms ? tiles : 2 * h->sms;  // two CTAs per SM
    // the curve volume as a 3D tensor (words along x, disparity group, row)
    // for the kernel's per-tile block loads
    CUtensorMap tm_curve;
    const uint64_t dims[3] = {uint64_t(a.W) + 2, uint64_t(inf::kGroups), uint64_t(a.H)};
    const uint64_t strides[2] = {curves->pitch_bytes, curves->pitch_bytes * inf::kGroups};
    const uint32_t box[3] = {uint32_t(inf::kBoxWords), uint32_t(inf::kGroups), 1};
    if (int rc = make_tmap_nd(&tm_curve, curves->ptr, CU_TENSOR_MAP_DATA_TYPE_UINT32, 4, 3, dims, strides, box))
        return rc;
    // programmatic stream serialisation: the kernel's prologue (weight
    // image, barriers, TMEM) overlaps the tail of the previous kernel on the
    // stream; griddepcontrol.wait in the kernel orders the data
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(inf::kNT);
    cfg.dynamicSmemBytes = inf::kSmem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CT_CUDA_TRY(cudaLaunchKernelEx(&cfg, inf::infer_kernel, tm_curve, a));
    CT_LAUNCH_CHECK();
    return CT_OK;
}

}  // extern "C"
