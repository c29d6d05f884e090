// crosscheck.cu — CrossCheckDisparityMaps::CDriver.
//
// Per pixel (CrossCheckDisparityMaps.cu:63-110): a base pixel holding a
// disparity code v = d + First is kept iff x -/+ d lies inside the image and
// the other map's code there is within disp_delta_thresh of v, compared as
// raw codes (.cu:94: an ID or Unknown in the other map is compared by its
// value too); otherwise it becomes Inconsistent. Non-disparity codes are
// copied through. U8 maps (a library format; 0xFF = not a disparity) keep d
// only against a disparity of the other map. The driver leaves the result's
// 1-pixel frame unwritten and out of the range, as the reference kernel does
// (.cu:71, IsInside(x, y, 1, 1)); process_lr's checked map is written
// everywhere. The kept range is reduced on the device with one warp
// reduction and one atomic per warp, into a word pair that a memset clears
// (min is stored as INT_MAX - d so that both halves reduce with max). Rows
// are 16-byte aligned (checked at the C ABI), so each thread moves 16 bytes
// of the base and result rows with one load and one store.
#include "ct_internal.h"
#include "ct_device.cuh"

namespace ct {

namespace {

template <typename T>
__device__ __forceinline__ bool decode(T v, int& d);

template <>
__device__ __forceinline__ bool decode<uint8_t>(uint8_t v, int& d) {
    d = v;
    return v != 0xFF;
}
template <>
__device__ __forceinline__ bool decode<uint16_t>(uint16_t v, int& d) {
    d = int(v) - 1;
    return v >= CT_DISP_FIRST && v <= CT_DISP_LAST;
}

template <typename T>
__device__ __forceinline__ T inconsistent();
template <>
__device__ __forceinline__ uint8_t inconsistent<uint8_t>() { return 0xFF; }
template <>
__device__ __forceinline__ uint16_t inconsistent<uint16_t>() { return CT_DISP_INCONSISTENT; }

// One thread per 16 bytes of a row (16 U8 or 8 U16 pixels): one 16-byte
// load of the base row and one 16-byte store, the other map read where each
// disparity points (L1-cached).
// Whether the other map's code vo confirms base code v (disparity d).
template <typename T>
__device__ __forceinline__ bool confirms(T vo, T v, int d, int tol);
template <>
__device__ __forceinline__ bool confirms<uint8_t>(uint8_t vo, uint8_t, int d, int tol) {
    int dd;
    return decode<uint8_t>(vo, dd) && abs(dd - d) <= tol;
}
template <>
__device__ __forceinline__ bool confirms<uint16_t>(uint16_t vo, uint16_t v, int, int tol) {
    return abs(int(vo) - int(v)) <= tol;
}

// frame = 1: pixels of the 1-pixel image frame are neither written nor
// counted in the range (the reference driver's kernel skips them).
template <typename T>
__global__ void crosscheck_kernel(T* out, size_t po, const T* base, size_t pb, const T* other, size_t pt, int W,
                                  int H, int tol, int lr, int frame, int32_t* range) {
    constexpr int PX = 16 / sizeof(T);
    // launched with programmatic stream serialisation after the matcher
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int x0 = (blockIdx.x * blockDim.x + threadIdx.x) * PX;
    const int y = blockIdx.y;
    int kmin = 0x7FFFFFFF, kmax = -1;
    if (x0 < W && !(frame && (y == 0 || y == H - 1))) {
        const T* brow = reinterpret_cast<const T*>(reinterpret_cast<const char*>(base) + (size_t)y * pb);
        const T* orow = reinterpret_cast<const T*>(reinterpret_cast<const char*>(other) + (size_t)y * pt);
        T* rrow = reinterpret_cast<T*>(reinterpret_cast<char*>(out) + (size_t)y * po);
        // rows are 16-byte aligned, x0 a multiple of PX; a chunk holding a
        // frame column is stored pixel by pixel
        const int xa = frame ? 1 : 0, xb = frame ? W - 1 : W;  // written columns [xa, xb)
        const bool full = x0 >= xa && x0 + PX <= xb;
        union {
            uint4 q;
            T v[PX];
        } in, res;
        if (x0 + PX <= W) in.q = *reinterpret_cast<const uint4*>(brow + x0);
        else
            for (int i = 0; i < PX; ++i) in.v[i] = x0 + i < W ? brow[x0 + i] : T(0);
#pragma unroll
        for (int i = 0; i < PX; ++i) {
            const int x = x0 + i;
            const T v = in.v[i];
            T r = v;
            int d;
            if (decode<T>(v, d)) {
                const int xo = lr ? x - d : x + d;
                r = inconsistent<T>();
                if (xo >= 0 && xo < W && x >= xa && x < xb) {
                    if (confirms<T>(__ldg(orow + xo), v, d, tol)) {
                        r = v;
                        kmin = min(kmin, d);
                        kmax = max(kmax, d);
                    }
                }
            }
            res.v[i] = r;
        }
        if (full) *reinterpret_cast<uint4*>(rrow + x0) = res.q;
        else
            for (int i = 0; i < PX; ++i)
                if (x0 + i >= xa && x0 + i < xb) rrow[x0 + i] = res.v[i];
    }
    if (range) {
        const unsigned mn = __reduce_max_sync(0xffffffffu, kmax >= 0 ? unsigned(0x7FFFFFFF - kmin) : 0u);
        const unsigned mx = __reduce_max_sync(0xffffffffu, unsigned(kmax + 1));
        if ((threadIdx.x & 31) == 0) {
            if (mn) atomicMax(reinterpret_cast<unsigned*>(&range[0]), mn);
            if (mx) atomicMax(reinterpret_cast<unsigned*>(&range[1]), mx);
        }
    }
}

struct CrossCheckHandle : ct_handle {
    CrossCheckHandle() : ct_handle(Kind::CrossCheck) {}
    ~CrossCheckHandle() override {
        if (device >= 0) cudaSetDevice(device);
        cudaFree(range);
    }
    ct_format fmt{};
    ct_crosscheck_params par{};
    int32_t* range = nullptr;  // [2] encoded min / max
};

}  // namespace

int crosscheck_launch(const ct_image* result, const ct_image* base, const ct_image* other, int tol, int lr,
                      int frame, int32_t* range, cudaStream_t s) {
    const int W = base->width, H = base->height;
    const int px = 16 / int(pix_size(base->type));  // pixels per thread
    dim3 grid((W + 128 * px - 1) / (128 * px), H);
    if (range) CT_CUDA_TRY(cudaMemsetAsync(range, 0, 2 * sizeof(int32_t), s));
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(128);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (base->type == CT_PIX_U8) {
        CT_CUDA_TRY(cudaLaunchKernelEx(&cfg, crosscheck_kernel<uint8_t>, static_cast<uint8_t*>(result->ptr),
                                       result->pitch_bytes, static_cast<const uint8_t*>(base->ptr), base->pitch_bytes,
                                       static_cast<const uint8_t*>(other->ptr), other->pitch_bytes, W, H, tol, lr,
                                       frame, range));
    } else {
        CT_CUDA_TRY(cudaLaunchKernelEx(&cfg, crosscheck_kernel<uint16_t>, static_cast<uint16_t*>(result->ptr),
                                       result->pitch_bytes, static_cast<const uint16_t*>(base->ptr), base->pitch_bytes,
                                       static_cast<const uint16_t*>(other->ptr), other->pitch_bytes, W, H, tol, lr,
                                       frame, range));
    }
    CT_LAUNCH_CHECK();
    return CT_OK;
}

}  // namespace ct

using namespace ct;

extern "C" {

int ct_crosscheck_create(ct_handle** out) {
    clear_error();
    if (!out) return fail(CT_EINVAL, "null output handle pointer");
    *out = new CrossCheckHandle();
    return CT_OK;
}

int ct_crosscheck_configure(ct_handle* hh, int32_t device, const ct_format* fmt, const ct_crosscheck_params* p) {
    clear_error();
    auto* h = (hh && hh->kind == Kind::CrossCheck) ? static_cast<CrossCheckHandle*>(hh) : nullptr;
    if (!h) return fail(CT_ESTATE, "not a cross-check handle");
    if (!fmt || !p) return fail(CT_EINVAL, "null format or parameters");
    if (fmt->type != CT_PIX_U8 && fmt->type != CT_PIX_U16)
        return fail(CT_ETYPE, "disparity maps must be U8 or U16");
    if (fmt->width < 1 || fmt->height < 1) return fail(CT_EINVAL, "bad size");
    if (p->disp_delta_thresh < 0) return fail(CT_EINVAL, "disp_delta_thresh must be >= 0");
    if (int rc = use_device(device)) return rc;
    h->device = device;
    if (int rc = h->init_status()) return rc;
    if (!h->range && cudaMalloc(&h->range, 2 * sizeof(int32_t)) != cudaSuccess)
        return fail(CT_ENOMEM, "range buffer");
    CT_CUDA_TRY(cudaMemset(h->range, 0, 2 * sizeof(int32_t)));
    h->fmt = *fmt;
    h->par = *p;
    h->configured = true;
    return CT_OK;
}

int ct_crosscheck_process(ct_handle* hh, const ct_image* result, const ct_image* disp_base,
                          const ct_image* disp_other, ct_stream stream) {
    clear_error();
    auto* h = (hh && hh->kind == Kind::CrossCheck) ? static_cast<CrossCheckHandle*>(hh) : nullptr;
    if (!h) return fail(CT_ESTATE, "not a cross-check handle");
    if (!h->configured) return fail(CT_ESTATE, "process before configure");
    const uint32_t t = 1u << h->fmt.type;
    if (int rc = check_image(disp_base, "disp_base", t)) return rc;
    if (int rc = check_image(disp_other, "disp_other", t)) return rc;
    if (int rc = check_image(result, "result", t)) return rc;
    if (int rc = check_same_size(disp_base, disp_other, "disp_base", "disp_other")) return rc;
    if (int rc = check_same_size(disp_base, result, "disp_base", "result")) return rc;
    if (disp_base->width != h->fmt.width || disp_base->height != h->fmt.height)
        return fail(CT_EFORMAT, "map size differs from the configured format");
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    return crosscheck_launch(result, disp_base, disp_other, h->par.disp_delta_thresh, h->par.left_to_right ? 1 : 0,
                             /*frame*/ 1, h->range, s);
}

int ct_crosscheck_range(ct_handle* hh, int32_t* disp_min, int32_t* disp_max) {
    clear_error();
    auto* h = (hh && hh->kind == Kind::CrossCheck) ? static_cast<CrossCheckHandle*>(hh) : nullptr;
    if (!h) return fail(CT_ESTATE, "not a cross-check handle");
    if (!disp_min || !disp_max) return fail(CT_EINVAL, "null output");
    if (!h->configured) return fail(CT_ESTATE, "range before configure");
    if (int rc = use_device(h->device)) return rc;
    if (h->last_stream) CT_CUDA_TRY(cudaStreamSynchronize(h->last_stream));
    else CT_CUDA_TRY(cudaDeviceSynchronize());
    uint32_t r[2];
    CT_CUDA_TRY(cudaMemcpy(r, h->range, sizeof r, cudaMemcpyDeviceToHost));
    *disp_min = r[0] ? int32_t(0x7FFFFFFF - r[0]) : INT32_MAX;
    *disp_max = int32_t(r[1]) - 1;
    return CT_OK;
}

}  // extern "C"
