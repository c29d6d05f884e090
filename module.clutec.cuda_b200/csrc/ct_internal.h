// ct_internal.h — host-side plumbing shared by the ctstereo C ABI:
// handle base class, error reporting, image validation, TMA descriptors.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/ctstereo.h"

namespace ct {

// Handle kinds (one per reference driver type).
enum class Kind : int32_t {
    Census = 1,
    BmCensus = 2,
    BmSad = 3,
    BmNcc = 4,
    BmAw = 5,
    CrossCheck = 6,
    Batch = 7,
    ConfNet = 8,
    Stream = 9,
    Map3D = 10,
    Compat = 11,
};

// Sets the thread-local message returned by ct_last_error_string and returns
// the code, so call sites read `return fail(CT_EINVAL, "...")`.
int fail(int code, const char* fmt, ...);
void clear_error();

#define CT_CUDA_TRY(expr)                                                          \
    do {                                                                           \
        cudaError_t e__ = (expr);                                                  \
        if (e__ != cudaSuccess)                                                    \
            return ::ct::fail(CT_ECUDA, "%s failed: %s (%s:%d)", #expr,            \
                              cudaGetErrorString(e__), __FILE__, __LINE__);        \
    } while (0)

// Launch check: a launch error (bad configuration) is reported right away;
// asynchronous faults surface at the next synchronising call.
#define CT_LAUNCH_CHECK()                                                          \
    do {                                                                           \
        cudaError_t e__ = cudaGetLastError();                                      \
        if (e__ != cudaSuccess)                                                    \
            return ::ct::fail(CT_ECUDA, "kernel launch failed: %s (%s:%d)",        \
                              cudaGetErrorString(e__), __FILE__, __LINE__);        \
    } while (0)

// Base of every handle. Holds the device, a device status word written by
// kernels whose bounded waits give up, and the last stream used.
struct Handle {
    Kind kind;
    int device = -1;
    bool configured = false;
    int32_t* d_status = nullptr;   // one int32 in device memory
    cudaStream_t last_stream = nullptr;
    float grad_thresh = 0.0f;      // gradient gate of the SAD / NCC / AW matchers (0: off)
    explicit Handle(Kind k) : kind(k) {}
    virtual ~Handle();
    int init_status();             // allocates d_status on the current device
};

// Element size of a pixel type; 0 if unknown.
size_t pix_size(int32_t type);

// Validates an image argument: non-null, known type in `allowed` (bit mask of
// 1 << type), pitch >= width * elem, positive size, 16-byte aligned pointer
// for vector access.
int check_image(const ct_image* im, const char* name, uint32_t allowed_types);
int check_same_size(const ct_image* a, const ct_image* b, const char* an, const char* bn);

// Makes `device` current and records it; returns CT_ECUDA on failure.
int use_device(int device);

// 2D TMA descriptor for a pitched buffer: element type / size, width x height
// elements, pitch in bytes, box = box_w x box_h elements. Out-of-bounds
// elements read as zero.
int make_tmap_2d(CUtensorMap* map, const void* base, CUtensorMapDataType dtype, size_t elem_bytes,
                 uint64_t width, uint64_t height, uint64_t pitch_bytes, uint32_t box_w, uint32_t box_h);

// Rank-N TMA descriptor (N <= 5): dims[0] innermost, strides_bytes[i] = byte
// stride of dimension i + 1, box[i] elements per dimension. Out-of-bounds
// elements read as zero.
int make_tmap_nd(CUtensorMap* map, const void* base, CUtensorMapDataType dtype, size_t elem_bytes, int rank,
                 const uint64_t* dims, const uint64_t* strides_bytes, const uint32_t* box);

// Device properties cached per device.
int sm_count(int device);

// Gradient gate on a finished disparity map (gate.cu): kind 0 = mean
// |I(x) - I(x+1)| over the P x P patch, 1 = standard deviation in percent;
// gated pixels become "no disparity" (and score 0). thresh <= 0: no-op.
int gate_launch(const ct_image* disp, const ct_image* score, const ct_image* base, int kind, int P, float thresh,
                cudaStream_t s);

}  // namespace ct

// Opaque handle type of the C ABI is the C++ base class.
struct ct_handle : ct::Handle {
    using ct::Handle::Handle;
};
