// map3d.cu — disparity to 3D points (MapDisparityTo3D::CDriver,
// MapDisparityTo3D.h:41-150 / MapDisparityTo3D.cu:75-330) with explicit
// pinhole cameras in place of the reference's _CStereoPinhole (CluTec.Core,
// not in the reference tree; the camera arithmetic is this library's own).
//
// One thread per pixel (HBM-bound: 1-4 B read, 16 B written): the left ray
// through (x, y) and the right ray through (x - d, y) are intersected at the
// midpoint of their closest points, computed from n = dL x dR as
// s = ((oR - oL) x dR) . n / |n|^2, t = ((oR - oL) x dL) . n / |n|^2 (no
// 1 - cos^2 cancellation for the nearly parallel rays of small
// disparities); rays with |n|^2 <= 1e-14 |dL|^2 |dR|^2 count as parallel.
// The range of the valid points is reduced per block (__reduce_min_sync on
// order-preserving integer keys, then shared memory) with at most one
// atomic per block and component, issued only when it can lower the stored
// key, instead of the reference's lock-guarded per-thread table
// (MapDisparityTo3D.cu:200-236).
#include "ct_internal.h"

#include <algorithm>
#include <cfloat>

namespace ct {
namespace m3d {

struct Cam {
    float fx, fy, cx, cy;
    float r[9];
    float c[3];
};

struct Params {
    int disp_min, disp_max;
    float sy, sz;  // output scale of Y and Z (-1 for the x-right, y-up, z-towards system)
    Cam cam[2];
};

// Order-preserving key of a float: a < b <=> key(a) < key(b).
__host__ __device__ inline uint32_t fkey(float f) {
    uint32_t u;
    memcpy(&u, &f, 4);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
inline float unkey(uint32_t k) {
    const uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

__device__ __forceinline__ float3 ray(const Cam& k, float x, float y) {
    const float u = __fdiv_rn(x - k.cx, k.fx), v = __fdiv_rn(y - k.cy, k.fy);
    return make_float3(k.r[0] * u + k.r[1] * v + k.r[2], k.r[3] * u + k.r[4] * v + k.r[5],
                       k.r[6] * u + k.r[7] * v + k.r[8]);
}

__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Disparity code of pixel x of a row: U16 as stored, U8 d -> d + 1 (255 ->
// CannotEvaluate), F32 d >= 0 -> d + 1 (sub-pixel; negative -> CannotEvaluate).
template <typename T>
__device__ __forceinline__ float code_of(const T* row, int x) {
    const T v = row[x];
    if constexpr (sizeof(T) == 1) return v == 0xFF ? float(CT_DISP_CANNOT_EVALUATE) : float(v) + 1.f;
    else if constexpr (sizeof(T) == 2) return float(v);
    else return v >= 0.f ? v + 1.f : float(CT_DISP_CANNOT_EVALUATE);
}

// range[0..2]: min keys of x, y, z; range[3..5]: min keys of -x, -y, -z (so
// one 0xFF fill initialises both halves).
template <typename T>
__global__ void __launch_bounds__(256) map3d_kernel(float4* out, size_t opitch, const T* disp, size_t dpitch, int W,
                                                     int H, Params p, uint32_t* range) {
    // blocks stride over the rows (grid y is a few blocks per SM), so the
    // range is reduced once per block
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t k[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu};
    for (int y = blockIdx.y; y < H && x < W; y += gridDim.y) {
        const T* drow = reinterpret_cast<const T*>(reinterpret_cast<const char*>(disp) + (size_t)y * dpitch);
        const float code = code_of(drow, x);
        const bool valid = code >= float(p.disp_min) && code <= float(p.disp_max);
        // (a sub-pixel map's disparity is used as stored, not through its code)
        const float d = valid ? (sizeof(T) == 4 ? float(drow[x]) : code - 1.f) : float(p.disp_min);
        const float3 dl = ray(p.cam[0], float(x), float(y));
        const float3 dr = ray(p.cam[1], float(x) - d, float(y));
        const float3 n = cross(dl, dr);
        const float nn = dot(n, n);
        const bool hit = nn > 1e-14f * dot(dl, dl) * dot(dr, dr);
        float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
        if (hit) {
            const float3 b = make_float3(p.cam[1].c[0] - p.cam[0].c[0], p.cam[1].c[1] - p.cam[0].c[1],
                                         p.cam[1].c[2] - p.cam[0].c[2]);
            const float s = __fdiv_rn(dot(cross(b, dr), n), nn);
            const float t = __fdiv_rn(dot(cross(b, dl), n), nn);
            float3 P = make_float3(0.5f * ((p.cam[0].c[0] + s * dl.x) + (p.cam[1].c[0] + t * dr.x)),
                                   0.5f * ((p.cam[0].c[1] + s * dl.y) + (p.cam[1].c[1] + t * dr.y)),
                                   0.5f * ((p.cam[0].c[2] + s * dl.z) + (p.cam[1].c[2] + t * dr.z)));
            P.y *= p.sy;
            P.z *= p.sz;
            o = make_float4(P.x, P.y, P.z, valid ? 1.f : 0.f);
            if (valid) {
                k[0] = min(k[0], fkey(P.x));
                k[1] = min(k[1], fkey(P.y));
                k[2] = min(k[2], fkey(P.z));
                k[3] = min(k[3], fkey(-P.x));
                k[4] = min(k[4], fkey(-P.y));
                k[5] = min(k[5], fkey(-P.z));
            }
        }
        reinterpret_cast<float4*>(reinterpret_cast<char*>(out) + (size_t)y * opitch)[x] = o;
    }
    // warp minima -> block minima -> one atomic per component, and only when
    // the stored key is larger (it only decreases, so a stale read can only
    // cause an unneeded atomic, never a missed one)
    __shared__ uint32_t red[256 / 32][6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const uint32_t m = __reduce_min_sync(0xffffffffu, k[i]);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][i] = m;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        uint32_t m = red[0][threadIdx.x];
#pragma unroll
        for (int w = 1; w < 256 / 32; ++w) m = min(m, red[w][threadIdx.x]);
        if (m != 0xFFFFFFFFu && m < *reinterpret_cast<volatile uint32_t*>(&range[threadIdx.x]))
            atomicMin(&range[threadIdx.x], m);
    }
}

}  // namespace m3d

namespace {

struct Map3DHandle : ct_handle {
    Map3DHandle() : ct_handle(Kind::Map3D) {}
    ~Map3DHandle() override {
        if (device >= 0) cudaSetDevice(device);
        cudaFree(range);
    }
    ct_format fmt{};
    m3d::Params par{};
    uint32_t* range = nullptr;  // [8]: 6 keys used
};

Map3DHandle* as_map3d(ct_handle* h) {
    return (h && h->kind == Kind::Map3D) ? static_cast<Map3DHandle*>(h) : nullptr;
}

}  // namespace
}  // namespace ct

using namespace ct;

extern "C" {

int ct_map3d_create(ct_handle** out) {
    clear_error();
    if (!out) return fail(CT_EINVAL, "null output handle pointer");
    *out = new Map3DHandle();
    return CT_OK;
}

int ct_map3d_configure(ct_handle* hh, int32_t device, const ct_format* fmt, const ct_map3d_params* p) {
    clear_error();
    Map3DHandle* h = as_map3d(hh);
    if (!h) return fail(CT_ESTATE, "not a disparity-to-3D handle");
    if (!fmt || !p) return fail(CT_EINVAL, "null format or parameters");
    if (fmt->type != CT_PIX_U8 && fmt->type != CT_PIX_U16 && fmt->type != CT_PIX_F32)
        return fail(CT_ETYPE, "disparity maps must be U8, U16 or F32");
    if (fmt->width < 1 || fmt->height < 1) return fail(CT_EINVAL, "bad size");
    if (p->reserved != 0) return fail(CT_EINVAL, "reserved field must be 0");
    if (p->disp_min > p->disp_max) return fail(CT_EINVAL, "disp_min above disp_max");
    for (int c = 0; c < 2; ++c)
        if (!(p->cam[c].fx != 0.f) || !(p->cam[c].fy != 0.f))
            return fail(CT_EINVAL, "camera %d: focal lengths must be non-zero", c);
    if (int rc = use_device(device)) return rc;
    h->device = device;
    if (int rc = h->init_status()) return rc;
    if (!h->range && cudaMalloc(&h->range, 8 * sizeof(uint32_t)) != cudaSuccess)
        return fail(CT_ENOMEM, "range buffer");
    CT_CUDA_TRY(cudaMemset(h->range, 0xFF, 8 * sizeof(uint32_t)));
    h->fmt = *fmt;
    m3d::Params k{};
    k.disp_min = p->disp_min;
    k.disp_max = p->disp_max;
    k.sy = p->cs_rut ? -1.f : 1.f;
    k.sz = p->cs_rut ? -1.f : 1.f;
    for (int c = 0; c < 2; ++c) {
        const ct_pinhole& q = p->cam[c];
        k.cam[c] = m3d::Cam{q.fx, q.fy, q.cx, q.cy, {}, {q.center[0], q.center[1], q.center[2]}};
        for (int i = 0; i < 9; ++i) k.cam[c].r[i] = q.rot[i];
    }
    h->par = k;
    h->configured = true;
    return CT_OK;
}

int ct_map3d_process(ct_handle* hh, const ct_image* map3d, const ct_image* disp, ct_stream stream) {
    clear_error();
    Map3DHandle* h = as_map3d(hh);
    if (!h) return fail(CT_ESTATE, "not a disparity-to-3D handle");
    if (!h->configured) return fail(CT_ESTATE, "process before configure");
    if (int rc = check_image(disp, "disp", 1u << h->fmt.type)) return rc;
    if (int rc = check_image(map3d, "map3d", 1u << CT_PIX_F32X4)) return rc;
    if (int rc = check_same_size(map3d, disp, "map3d", "disp")) return rc;
    if (disp->width != h->fmt.width || disp->height != h->fmt.height)
        return fail(CT_EFORMAT, "map size differs from the configured format");
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    CT_CUDA_TRY(cudaMemsetAsync(h->range, 0xFF, 8 * sizeof(uint32_t), s));
    const int gx = (disp->width + 255) / 256;
    const int gy = std::max(1, std::min(disp->height, 8 * sm_count(h->device) / gx));
    const dim3 grid(gx, gy);
    float4* out = static_cast<float4*>(map3d->ptr);
    if (disp->type == CT_PIX_U8)
        m3d::map3d_kernel<uint8_t><<<grid, 256, 0, s>>>(out, map3d->pitch_bytes, static_cast<const uint8_t*>(disp->ptr),
                                                        disp->pitch_bytes, disp->width, disp->height, h->par, h->range);
    else if (disp->type == CT_PIX_U16)
        m3d::map3d_kernel<uint16_t><<<grid, 256, 0, s>>>(out, map3d->pitch_bytes,
                                                         static_cast<const uint16_t*>(disp->ptr), disp->pitch_bytes,
                                                         disp->width, disp->height, h->par, h->range);
    else
        m3d::map3d_kernel<float><<<grid, 256, 0, s>>>(out, map3d->pitch_bytes, static_cast<const float*>(disp->ptr),
                                                      disp->pitch_bytes, disp->width, disp->height, h->par, h->range);
    CT_LAUNCH_CHECK();
    return CT_OK;
}

int ct_map3d_range(ct_handle* hh, float* min_xyz, float* max_xyz) {
    clear_error();
    Map3DHandle* h = as_map3d(hh);
    if (!h) return fail(CT_ESTATE, "not a disparity-to-3D handle");
    if (!min_xyz || !max_xyz) return fail(CT_EINVAL, "null output");
    if (!h->configured) return fail(CT_ESTATE, "range before configure");
    if (int rc = use_device(h->device)) return rc;
    if (h->last_stream) CT_CUDA_TRY(cudaStreamSynchronize(h->last_stream));
    else CT_CUDA_TRY(cudaDeviceSynchronize());
    uint32_t k[8];
    CT_CUDA_TRY(cudaMemcpy(k, h->range, sizeof k, cudaMemcpyDeviceToHost));
    for (int i = 0; i < 3; ++i) {
        const bool none = k[i] == 0xFFFFFFFFu;  // no valid point (ResetRange's values)
        min_xyz[i] = none ? FLT_MAX : m3d::unkey(k[i]);
        max_xyz[i] = none ? -FLT_MAX : -m3d::unkey(k[3 + i]);
    }
    return CT_OK;
}

}  // extern "C"
