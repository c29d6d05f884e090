// color.cu — disparity visualisation (ColorDisparityImage::CDriver,
// ColorDisparityImage.h:37-120 / ColorDisparityImage.cu:45-300), written into
// a headless device image (RGBA8 or U16) instead of a GL surface.
//
// A map entry is read as an EDisparityId code: U16 maps as they are, U8 maps
// as d + 1 (255 -> CannotEvaluate). With t = (code - disp_min) / (disp_max -
// disp_min) in FP32 (IEEE division) and q(t, M) = rint(clamp(t, 0, 1) * M):
//   ANALYSIS  RGBA8: disparities gray (q(t, 255) in r, g, b), every other
//             code its colour from the parameter table, unknown codes red
//   GRAY      U16: disparities q(t, 65535), others 0
//   COLOR     RGBA8: disparities on the blue-green-red ramp of
//             NormFloatToColor (Conversion.h:56-74): b = 1 - min(t / 0.7, 1),
//             g = 1 - min(|t - 0.5| / 0.59, 1), r = 1 - min(|t - 0.8| / 0.7, 1),
//             each divided by the largest of the three, then q(., 255);
//             others black (alpha 255)
//   DISP_ABS  U16: disparities their code, others 0
//   DISP_REL  U16: disparities (0x7FFF + inf_offset) - (code - First), others 0
// One thread per pixel; the kernel is HBM-bound (read 1-2 B, write 2-4 B).
#include "ct_internal.h"

namespace ct {
namespace color {

struct Params {
    int style, disp_min, disp_max, inf_offset;
    uint32_t colors[7];  // RGBA8 (r in the low byte): unknown, cannot evaluate, saturated, not specific,
                         // not found, not unique, inconsistent
};

__device__ __forceinline__ uint32_t q(float t, float M) { return uint32_t(rintf(fminf(fmaxf(t, 0.f), 1.f) * M)); }

__device__ __forceinline__ uint32_t rgba(uint32_t r, uint32_t g, uint32_t b) { return r | (g << 8) | (b << 16) | 0xFF000000u; }

__global__ void color_kernel(const void* disp, size_t dpitch, int dtype, void* out, size_t opitch, int W, int H,
                             Params p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const char* drow = static_cast<const char*>(disp) + (size_t)y * dpitch;
    uint32_t code;
    if (dtype == CT_PIX_U8) {
        const uint32_t v = reinterpret_cast<const uint8_t*>(drow)[x];
        code = v == 0xFFu ? CT_DISP_CANNOT_EVALUATE : v + 1;
    } else {
        code = reinterpret_cast<const uint16_t*>(drow)[x];
    }
    const bool is_disp = code >= CT_DISP_FIRST && code <= CT_DISP_LAST;
    const float t = __fdiv_rn(float(int(code) - p.disp_min), float(p.disp_max - p.disp_min));
    char* orow = static_cast<char*>(out) + (size_t)y * opitch;
    switch (p.style) {
        case CT_COLOR_ANALYSIS: {
            uint32_t c;
            if (is_disp) {
                const uint32_t g = q(t, 255.f);
                c = rgba(g, g, g);
            } else {
                switch (code) {
                    case CT_DISP_UNKNOWN: c = p.colors[0]; break;
                    case CT_DISP_CANNOT_EVALUATE: c = p.colors[1]; break;
                    case CT_DISP_SATURATED: c = p.colors[2]; break;
                    case CT_DISP_NOT_SPECIFIC: c = p.colors[3]; break;
                    case CT_DISP_NOT_FOUND: c = p.colors[4]; break;
                    case CT_DISP_NOT_UNIQUE: c = p.colors[5]; break;
                    case CT_DISP_INCONSISTENT: c = p.colors[6]; break;
                    default: c = rgba(255, 0, 0); break;
                }
            }
            reinterpret_cast<uint32_t*>(orow)[x] = c;
            break;
        }
        case CT_COLOR_COLOR: {
            uint32_t c = rgba(0, 0, 0);
            if (is_disp) {
                const float fb = 1.f - fminf(__fdiv_rn(t, 0.7f), 1.f);
                const float fg = 1.f - fminf(__fdiv_rn(fabsf(t - 0.5f), 0.59f), 1.f);
                const float fr = 1.f - fminf(__fdiv_rn(fabsf(t - 0.8f), 0.7f), 1.f);
                const float fm = fmaxf(fmaxf(fr, fg), fb);
                c = rgba(q(__fdiv_rn(fr, fm), 255.f), q(__fdiv_rn(fg, fm), 255.f), q(__fdiv_rn(fb, fm), 255.f));
            }
            reinterpret_cast<uint32_t*>(orow)[x] = c;
            break;
        }
        case CT_COLOR_GRAY:
            reinterpret_cast<uint16_t*>(orow)[x] = is_disp ? uint16_t(q(t, 65535.f)) : uint16_t(0);
            break;
        case CT_COLOR_DISP_ABS:
            reinterpret_cast<uint16_t*>(orow)[x] = is_disp ? uint16_t(code) : uint16_t(0);
            break;
        default:  // CT_COLOR_DISP_REL
            reinterpret_cast<uint16_t*>(orow)[x] =
                is_disp ? uint16_t(uint32_t(0x7FFF + p.inf_offset) - (code - CT_DISP_FIRST)) : uint16_t(0);
            break;
    }
}

}  // namespace color
}  // namespace ct

using namespace ct;

extern "C" {

int ct_color_disparity(const ct_image* out, const ct_image* disp, const ct_color_params* p, ct_stream stream) {
    clear_error();
    if (!p) return fail(CT_EINVAL, "null parameters");
    if (p->style < CT_COLOR_ANALYSIS || p->style > CT_COLOR_DISP_REL) return fail(CT_EINVAL, "unknown style");
    if ((p->style == CT_COLOR_GRAY || p->style == CT_COLOR_COLOR || p->style == CT_COLOR_ANALYSIS) &&
        p->disp_max <= p->disp_min)
        return fail(CT_EINVAL, "disp_max must exceed disp_min");
    if (int rc = check_image(disp, "disp", (1u << CT_PIX_U8) | (1u << CT_PIX_U16))) return rc;
    const bool rgba = p->style == CT_COLOR_ANALYSIS || p->style == CT_COLOR_COLOR;
    if (int rc = check_image(out, "out", 1u << (rgba ? CT_PIX_RGBA8 : CT_PIX_U16))) return rc;
    if (int rc = check_same_size(out, disp, "out", "disp")) return rc;
    color::Params k{p->style, p->disp_min, p->disp_max, p->inf_offset, {}};
    for (int i = 0; i < 7; ++i) k.colors[i] = p->colors[i];
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    color::color_kernel<<<dim3((disp->width + 255) / 256, disp->height), 256, 0, s>>>(
        disp->ptr, disp->pitch_bytes, disp->type, out->ptr, out->pitch_bytes, disp->width, disp->height, k);
    CT_LAUNCH_CHECK();
    return CT_OK;
}

int ct_color_params_default(int32_t style, ct_color_params* p) {
    clear_error();
    if (!p) return fail(CT_EINVAL, "null output");
    *p = ct_color_params{};
    p->style = style;
    p->disp_min = CT_DISP_FIRST;
    p->disp_max = CT_DISP_LAST;
    p->inf_offset = 0;
    // SParameter's defaults (ColorDisparityImage.h:75-87), RGBA8 with r in the low byte
    const uint8_t c[7][3] = {{10, 100, 180}, {0, 150, 50}, {0, 200, 200}, {200, 0, 200},
                             {200, 50, 50}, {240, 50, 150}, {100, 10, 10}};
    for (int i = 0; i < 7; ++i) p->colors[i] = uint32_t(c[i][0]) | (uint32_t(c[i][1]) << 8) | (uint32_t(c[i][2]) << 16) | 0xFF000000u;
    return CT_OK;
}

}  // extern "C"
