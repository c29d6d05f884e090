// common.cpp — host plumbing: errors, handle base, validation, TMA descriptors.
#include "ct_internal.h"

#include <mutex>
#include <vector>

namespace ct {

namespace {
thread_local std::string g_last_error;
}

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

void clear_error() { g_last_error.clear(); }

Handle::~Handle() {
    if (d_status) {
        int prev = -1;
        cudaGetDevice(&prev);
        if (device >= 0) cudaSetDevice(device);
        cudaFree(d_status);
        if (prev >= 0) cudaSetDevice(prev);
    }
}

int Handle::init_status() {
    if (d_status) return CT_OK;
    if (cudaMalloc(&d_status, sizeof(int32_t)) != cudaSuccess)
        return fail(CT_ENOMEM, "cudaMalloc of the status word failed");
    CT_CUDA_TRY(cudaMemset(d_status, 0, sizeof(int32_t)));
    return CT_OK;
}

size_t pix_size(int32_t type) {
    switch (type) {
        case CT_PIX_U8: return 1;
        case CT_PIX_U16: return 2;
        case CT_PIX_U64: return 8;
        case CT_PIX_F32: return 4;
        case CT_PIX_RGBA8: return 4;
        case CT_PIX_F32X4: return 16;
        case CT_PIX_U16X4: return 8;
        default: return 0;
    }
}

int check_image(const ct_image* im, const char* name, uint32_t allowed_types) {
    if (!im) return fail(CT_EINVAL, "%s: null image", name);
    if (!im->ptr) return fail(CT_EINVAL, "%s: null device pointer", name);
    if (im->type < 0 || im->type > 31 || !(allowed_types & (1u << im->type)))
        return fail(CT_ETYPE, "%s: pixel type %d not supported here", name, im->type);
    if (im->width <= 0 || im->height <= 0)
        return fail(CT_EINVAL, "%s: bad size %dx%d", name, im->width, im->height);
    if (im->pitch_bytes < (size_t)im->width * pix_size(im->type))
        return fail(CT_EINVAL, "%s: pitch %zu smaller than a row", name, im->pitch_bytes);
    if ((reinterpret_cast<uintptr_t>(im->ptr) & 15) != 0 || (im->pitch_bytes & 15) != 0)
        return fail(CT_EINVAL, "%s: pointer and pitch must be 16-byte aligned", name);
    if (im->reserved != 0) return fail(CT_EINVAL, "%s: reserved field must be 0", name);
    return CT_OK;
}

int check_same_size(const ct_image* a, const ct_image* b, const char* an, const char* bn) {
    if (a->width != b->width || a->height != b->height)
        return fail(CT_EFORMAT, "%s (%dx%d) and %s (%dx%d) do not have the same format", an, a->width,
                    a->height, bn, b->width, b->height);
    return CT_OK;
}

int use_device(int device) {
    int n = 0;
    CT_CUDA_TRY(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) return fail(CT_EINVAL, "device %d out of range (%d devices)", device, n);
    CT_CUDA_TRY(cudaSetDevice(device));
    return CT_OK;
}

namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;
}  // namespace

int make_tmap_2d(CUtensorMap* map, const void* base, CUtensorMapDataType dtype, size_t elem_bytes,
                 uint64_t width, uint64_t height, uint64_t pitch_bytes, uint32_t box_w, uint32_t box_h) {
    std::call_once(g_encode_once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!g_encode) return fail(CT_ECUDA, "cuTensorMapEncodeTiled is not available from the driver");
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (pitch_bytes & 15) || ((box_w * elem_bytes) & 15))
        return fail(CT_EINVAL, "TMA alignment: base, pitch and box row must be multiples of 16 bytes");
    cuuint64_t dims[2] = {width, height};
    cuuint64_t strides[1] = {pitch_bytes};
    cuuint32_t box[2] = {box_w, box_h};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(map, dtype, 2, const_cast<void*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(CT_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return CT_OK;
}

int make_tmap_nd(CUtensorMap* map, const void* base, CUtensorMapDataType dtype, size_t elem_bytes, int rank,
                 const uint64_t* dims, const uint64_t* strides_bytes, const uint32_t* box) {
    std::call_once(g_encode_once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!g_encode) return fail(CT_ECUDA, "cuTensorMapEncodeTiled is not available from the driver");
    if (rank < 1 || rank > 5) return fail(CT_EINVAL, "tensor rank %d", rank);
    if ((reinterpret_cast<uintptr_t>(base) & 15) || ((box[0] * elem_bytes) & 15))
        return fail(CT_EINVAL, "TMA alignment: base and box row must be multiples of 16 bytes");
    cuuint64_t d[5], st[4];
    cuuint32_t b[5], es[5];
    for (int i = 0; i < rank; ++i) {
        d[i] = dims[i];
        b[i] = box[i];
        es[i] = 1;
        if (i + 1 < rank) {
            st[i] = strides_bytes[i];
            if (st[i] & 15) return fail(CT_EINVAL, "TMA stride %d not a multiple of 16 bytes", i);
        }
    }
    CUresult r = g_encode(map, dtype, cuuint32_t(rank), const_cast<void*>(base), d, st, b, es,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(CT_ECUDA, "cuTensorMapEncodeTiled (rank %d) failed (%d)", rank, (int)r);
    return CT_OK;
}

int sm_count(int device) {
    static std::mutex mu;
    static std::vector<int> cache;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)cache.size() <= device) cache.resize(device + 1, 0);
    if (!cache[device]) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
        cache[device] = v > 0 ? v : 1;
    }
    return cache[device];
}

}  // namespace ct

extern "C" {

const char* ct_last_error_string(void) { return ct::g_last_error.c_str(); }

const char* ct_version(void) { return "ctstereo 0.1.0 sm_100a"; }

int ct_destroy(ct_handle* h) {
    ct::clear_error();
    delete h;
    return CT_OK;
}

int ct_bm_set_gradient_gate(ct_handle* h, float grad_thresh) {
    ct::clear_error();
    if (!h) return ct::fail(CT_EINVAL, "null handle");
    if (h->kind != ct::Kind::BmSad && h->kind != ct::Kind::BmNcc && h->kind != ct::Kind::BmAw)
        return ct::fail(CT_ESTATE, "the gradient gate belongs to the SAD, NCC and AW matchers");
    if (!(grad_thresh >= 0.0f)) return ct::fail(CT_EINVAL, "grad_thresh must be >= 0");
    h->grad_thresh = grad_thresh;
    return CT_OK;
}

int ct_handle_device_status(ct_handle* h, int32_t* status) {
    ct::clear_error();
    if (!h || !status) return ct::fail(CT_EINVAL, "null argument");
    *status = 0;
    if (!h->d_status) return CT_OK;
    if (int rc = ct::use_device(h->device)) return rc;
    if (h->last_stream) CT_CUDA_TRY(cudaStreamSynchronize(h->last_stream));
    else CT_CUDA_TRY(cudaDeviceSynchronize());
    int32_t v = 0;
    CT_CUDA_TRY(cudaMemcpy(&v, h->d_status, sizeof v, cudaMemcpyDeviceToHost));
    CT_CUDA_TRY(cudaMemset(h->d_status, 0, sizeof v));
    *status = v;
    return CT_OK;
}

}  // extern "C"
