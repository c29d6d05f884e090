// noalloc.cu — census matching that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code that runs while a stream is being
// captured into a CUDA graph, real-time loops whose allocator is frozen after
// start-up, or hosts whose device memory is owned by another framework's
// pool. ct_bm_census_process_static serves them: it runs the same census
// transform and census matcher kernels as ct_bm_census_process, but its
// scratch (the census descriptors of both views, the disparity merge keys and
// a status word) lives in the file-scope __device__ arrays below instead of
// memory a handle allocates.
//
// Limits and rules:
//  * Images up to kStaticMaxPixels = 2,097,152 pixels counted with the row
//    rounded up to a multiple of 4 (1920 x 1080 fits); larger images are
//    rejected with CT_EINVAL. The arrays take 40 MiB + 256 B of device memory
//    on every GPU that loads this library's module, until the process exits.
//  * The first call on a device looks up the arrays' device addresses
//    (cudaGetSymbolAddress with that device current). Make that first call
//    before any stream capture begins.
//  * All calls share the arrays: calls whose work overlaps on the GPU (other
//    streams, other host threads) race and corrupt each other's results.
//    Serialise them, e.g. on one stream.
//  * The arrays keep the previous call's contents; the merge keys must start
//    at 0xFFFFFFFF, so every call whose disparities span more than one CTA
//    clears them first (cudaMemsetAsync, which allocates nothing; the
//    finalize kernel also resets every key it reads, the clear guards against
//    a call that was cut short).
//  * Bounded device waits that give up write CT_ETIMEOUT into the caller's
//    status word, or, when the caller passes none, into a static word that
//    ct_bm_census_static_status reads and clears.
//  * The looked-up addresses belong to the device's current CUDA context; if
//    that context changes (cudaDeviceReset, a new primary context), the next
//    call looks them up again.
#include "ct_internal.h"
#include "ct_device.cuh"
#include "census_match.cuh"

#include <mutex>
#include <vector>

namespace ct {
namespace census {
int launch9x7(const ct_image* src, uint64_t* dst, size_t dst_pitch_elems, int32_t* status, cudaStream_t s,
              int planar);
}

namespace {

constexpr size_t kStaticMaxPixels = size_t(1) << 21;

static __device__ __align__(256) uint64_t g_static_desc[2 * kStaticMaxPixels];
static __device__ __align__(256) uint32_t g_static_keys[kStaticMaxPixels];
static __device__ __align__(256) int32_t g_static_status[64];

struct StaticScratch {
    CUcontext ctx = nullptr;  // context the addresses were looked up in
    uint64_t* desc = nullptr;
    uint32_t* keys = nullptr;
    int32_t* status = nullptr;
};

std::mutex g_mu;
std::vector<StaticScratch> g_scratch;  // by device ordinal

// The current context of this thread through the driver's entry point (the
// library does not link libcuda directly); NULL if none is bound yet.
CUcontext current_context() {
    static PFN_cuCtxGetCurrent_v4000 get = nullptr;
    if (!get) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        get = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(fn);
    }
    CUcontext ctx = nullptr;
    return get(&ctx) == CUDA_SUCCESS ? ctx : nullptr;
}

// Device addresses of the arrays on `device` (which is current). Host code
// must not pass the symbols themselves to a kernel: on the host they name a
// host-side shadow, not device memory.
int static_scratch(int device, StaticScratch* out) {
    std::lock_guard<std::mutex> lk(g_mu);
    if ((int)g_scratch.size() <= device) g_scratch.resize(device + 1);
    StaticScratch& s = g_scratch[device];
    // NULL before the runtime has bound a context to this thread; the lookup
    // below binds the device's primary context.
    CUcontext ctx = current_context();
    if (!s.desc || !ctx || s.ctx != ctx) {
        StaticScratch t;
        CT_CUDA_TRY(cudaGetSymbolAddress(reinterpret_cast<void**>(&t.desc), g_static_desc));
        CT_CUDA_TRY(cudaGetSymbolAddress(reinterpret_cast<void**>(&t.keys), g_static_keys));
        CT_CUDA_TRY(cudaGetSymbolAddress(reinterpret_cast<void**>(&t.status), g_static_status));
        CT_CUDA_TRY(cm::prepare_census_match());  // function attributes only
        t.ctx = current_context();
        s = t;
    }
    *out = s;
    return CT_OK;
}

}  // namespace
}  // namespace ct

using namespace ct;

extern "C" int ct_bm_census_process_static(const ct_image* disp, const ct_image* left, const ct_image* right,
                                           int32_t disp_count, int32_t left_to_right, int32_t* device_status,
                                           ct_stream stream) {
    clear_error();
    if (int rc = check_image(left, "left", 1u << CT_PIX_U8)) return rc;
    if (int rc = check_image(right, "right", 1u << CT_PIX_U8)) return rc;
    if (int rc = check_same_size(left, right, "left", "right")) return rc;
    if (int rc = check_image(disp, "disp", (1u << CT_PIX_U8) | (1u << CT_PIX_U16))) return rc;
    if (int rc = check_same_size(disp, left, "disp", "left")) return rc;
    const int W = left->width, H = left->height;
    if (W < 8 || H < 8) return fail(CT_EINVAL, "image size %dx%d below 8x8", W, H);
    if (disp_count < 1 || disp_count > 256) return fail(CT_EINVAL, "disp_count must be 1..256");
    if (disp->type == CT_PIX_U8 && disp_count > 255) return fail(CT_ETYPE, "U8 maps need disp_count <= 255");
    const size_t pitch = cm::planar_pitch(W);  // descriptor row (pair-planar layout), elements
    if (pitch * (size_t)H > kStaticMaxPixels)
        return fail(CT_EINVAL,
                    "image %dx%d exceeds the static scratch of ct_bm_census_process_static "
                    "(%zu pixels with rows rounded up to a multiple of 4; 1920x1080 fits)",
                    W, H, kStaticMaxPixels);
    int device = 0;
    CT_CUDA_TRY(cudaGetDevice(&device));
    StaticScratch sc;
    if (int rc = static_scratch(device, &sc)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int32_t* status = device_status ? device_status : sc.status;

    using namespace cm;
    uint64_t* dl = sc.desc;
    uint64_t* dr = sc.desc + pitch * H;
    if (disp_count > kDPC)  // the keys merge several disparity CTAs
        CT_CUDA_TRY(cudaMemsetAsync(sc.keys, 0xFF, (size_t)W * H * sizeof(uint32_t), s));
    if (int rc = census::launch9x7(left, dl, pitch, status, s, 1)) return rc;
    if (int rc = census::launch9x7(right, dr, pitch, status, s, 1)) return rc;
    const int dir = left_to_right ? 0 : 1;
    CUtensorMap tb, tm;
    if (int rc = make_planar_maps(&tb, &tm, dir == 0 ? dl : dr, dir == 0 ? dr : dl, W, H)) return rc;
    MatchArgs a{};
    a.W = W; a.H = H; a.D = disp_count;
    a.th = pick_strip_height(W, H, disp_count, sm_count(device));
    a.keys = sc.keys;
    a.merge_last = 0;  // one key plane merged by atomicMin (keeps the static scratch at 40 MiB)
    a.out = disp->ptr; a.out_pitch = disp->pitch_bytes; a.out_type = disp->type;
    a.status = status;
    const cudaError_t e = dir == 0 ? launch_census_match<0>(tb, tm, a, s) : launch_census_match<1>(tb, tm, a, s);
    if (e != cudaSuccess) return fail(CT_ECUDA, "census match launch failed: %s", cudaGetErrorString(e));
    return CT_OK;
}

extern "C" int ct_bm_census_static_status(int32_t* status) {
    clear_error();
    if (!status) return fail(CT_EINVAL, "null argument");
    *status = 0;
    int device = 0;
    CT_CUDA_TRY(cudaGetDevice(&device));
    StaticScratch sc;
    if (int rc = static_scratch(device, &sc)) return rc;
    CT_CUDA_TRY(cudaDeviceSynchronize());
    int32_t v = 0;
    CT_CUDA_TRY(cudaMemcpy(&v, sc.status, sizeof v, cudaMemcpyDeviceToHost));
    CT_CUDA_TRY(cudaMemset(sc.status, 0, sizeof v));
    *status = v;
    return CT_OK;
}
