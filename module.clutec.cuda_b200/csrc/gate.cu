// gate.cu — the reference matchers' gradient gate on the plain disparity maps.
//
// The reference drivers refuse to match patches with too little texture:
// EvalGrad marks them CannotEvaluate before the disparity search
// (BlockMatcherSAD1.cu:226-249 and BlockMatcherNCC.cu:388-413: the mean
// |I(x) - I(x+1)| over the patch; BlockMatcherAW1.cu:331-417: the patch's
// standard deviation, truncated to an integer, in percent of 255). The plain
// matchers here search every pixel and then apply the same test in one pass
// over the base image: a gated pixel's map entry becomes "no disparity"
// (U8 255, U16 CannotEvaluate, F32 -1) and its NCC score 0. The result is
// the map the reference's skip would give, since a gated pixel's search never
// influences another pixel.
#include "ct_internal.h"

namespace ct {
namespace gate {

constexpr int kTX = 32, kTY = 8;
constexpr int kMaxP = 13;

// kind 0: mean absolute horizontal gradient (SAD1, NCC); 1: standard
// deviation truncated to an integer, in percent (AW1). Patch [x - P/2,
// x - P/2 + P - 1]; I(x) = 0 beyond the right edge (SafeReadFromSurf's zero
// fill, Kernel.ArrayCache.h:278-293). Only pixels whose patch is inside the
// image are tested.
__global__ void gate_kernel(const uint8_t* img, size_t pitch, int W, int H, int kind, int P, float thresh,
                            void* out, size_t out_pitch, int out_type, float* score, size_t score_pitch) {
    __shared__ uint8_t t[kTY + kMaxP - 1][kTX + kMaxP + 3];
    const int pa = P / 2, pb = P - 1 - pa;
    const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY;
    const int RW = kTX + P, RH = kTY + P - 1;  // one extra column for the gradient
    for (int i = threadIdx.y * kTX + threadIdx.x; i < RW * RH; i += kTX * kTY) {
        const int r = i / RW, c = i % RW;
        const int xx = x0 - pa + c, yy = y0 - pa + r;
        t[r][c] = (xx >= 0 && xx < W && yy >= 0 && yy < H) ? img[(size_t)yy * pitch + xx] : 0;
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= W || y >= H || x - pa < 0 || x + pb >= W || y - pa < 0 || y + pb >= H) return;
    bool gated;
    if (kind == 0) {
        int g = 0;
        for (int r = 0; r < P; ++r)
            for (int c = 0; c < P; ++c)
                g += abs(int(t[threadIdx.y + r][threadIdx.x + c]) - int(t[threadIdx.y + r][threadIdx.x + c + 1]));
        gated = __fdiv_rn(__int2float_rn(g), __int2float_rn(P * P)) < thresh;
    } else {
        int s = 0, q = 0;
        for (int r = 0; r < P; ++r)
            for (int c = 0; c < P; ++c) {
                const int v = t[threadIdx.y + r][threadIdx.x + c];
                s += v;
                q += v * v;
            }
        const float fm = __fdiv_rn(__int2float_rn(s), __int2float_rn(P * P));
        const float fm2 = __fdiv_rn(__int2float_rn(q), __int2float_rn(P * P));
        const float sd = __fsqrt_rn(fabsf(__fsub_rn(fm2, __fmul_rn(fm, fm))));
        gated = __fmul_rn(__fdiv_rn(__int2float_rn(__float2int_rz(sd)), 255.0f), 100.0f) < thresh;
    }
    if (!gated) return;
    char* row = static_cast<char*>(out) + (size_t)y * out_pitch;
    if (out_type == CT_PIX_U8) reinterpret_cast<uint8_t*>(row)[x] = 0xFF;
    else if (out_type == CT_PIX_U16) reinterpret_cast<uint16_t*>(row)[x] = CT_DISP_CANNOT_EVALUATE;
    else reinterpret_cast<float*>(row)[x] = -1.0f;
    if (score) reinterpret_cast<float*>(reinterpret_cast<char*>(score) + (size_t)y * score_pitch)[x] = 0.0f;
}

}  // namespace gate

// Applies the gate to a finished map (and score). kind / P as gate_kernel;
// thresh <= 0 does nothing.
int gate_launch(const ct_image* disp, const ct_image* score, const ct_image* base, int kind, int P, float thresh,
                cudaStream_t s) {
    if (!(thresh > 0.0f)) return CT_OK;
    if (P < 1 || P > gate::kMaxP) return fail(CT_EINTERNAL, "gate patch %d out of range", P);
    const dim3 grid((base->width + gate::kTX - 1) / gate::kTX, (base->height + gate::kTY - 1) / gate::kTY);
    gate::gate_kernel<<<grid, dim3(gate::kTX, gate::kTY), 0, s>>>(
        static_cast<const uint8_t*>(base->ptr), base->pitch_bytes, base->width, base->height, kind, P, thresh,
        disp->ptr, disp->pitch_bytes, disp->type, score ? static_cast<float*>(score->ptr) : nullptr,
        score ? score->pitch_bytes : 0);
    CT_LAUNCH_CHECK();
    return CT_OK;
}

}  // namespace ct
