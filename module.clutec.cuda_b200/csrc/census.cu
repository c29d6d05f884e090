// census.cu — CensusTransform::CDriver and the census block matcher.
//
// Census transform (CensusTransform.cu:60-157): the 9x7 / 64-bit transform is
// census_tile.cuh; the 3x3 / 8-bit reference transform is kept for parity
// with the reference.
#include "ct_internal.h"
#include "ct_device.cuh"
#include "census_match.cuh"
#include "census_tile.cuh"

namespace ct {

// ---------------------------------------------------------------------------
// 9x7 census transform kernel
// ---------------------------------------------------------------------------
namespace census {

__global__ void __launch_bounds__(kNT) census9x7_kernel(const __grid_constant__ CUtensorMap tm_img, int W, int H,
                                                         uint64_t* out, size_t out_pitch_elems,
                                                         int32_t* status, int planar) {
    __shared__ __align__(128) TileSmem sm;
    // a matcher launched next with programmatic stream serialisation may
    // start its prologue now; it waits for these descriptors itself
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    census_tile(&tm_img, W, H, blockIdx.x * kTX, blockIdx.y * kTY, out, out_pitch_elems, planar, status, sm);
}

// Both views of a pair in one launch (blockIdx.z = view), so the tail wave
// of one view overlaps the other's tiles.
__global__ void __launch_bounds__(kNT) census9x7_pair_kernel(const __grid_constant__ CUtensorMap tm0,
                                                              const __grid_constant__ CUtensorMap tm1, int W, int H,
                                                              uint64_t* out0, uint64_t* out1, size_t out_pitch_elems,
                                                              int32_t* status, int planar) {
    __shared__ __align__(128) TileSmem sm;
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");  // as census9x7_kernel
    const bool second = blockIdx.z == 1;
    census_tile(second ? &tm1 : &tm0, W, H, blockIdx.x * kTX, blockIdx.y * kTY, second ? out1 : out0,
                out_pitch_elems, planar, status, sm);
}

// 3x3 / 8-bit reference transform (CensusTransform.cu:60-120): bits 7..0 =
// (-1,-1),(0,-1),(+1,-1),(-1,0),(+1,0),(-1,+1),(0,+1),(+1,+1), strict '>',
// 1-px border not written.
__global__ void census3x3_kernel(const uint8_t* img, size_t pitch, int W, int H, uint8_t* out,
                                 size_t out_pitch) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x < 1 || y < 1 || x >= W - 1 || y >= H - 1) return;
    auto P = [&](int dx, int dy) { return img[(size_t)(y + dy) * pitch + x + dx]; };
    const uint8_t c = P(0, 0);
    uint32_t v = 0;
    v |= 0x80u * (P(-1, -1) > c);
    v |= 0x40u * (P(0, -1) > c);
    v |= 0x20u * (P(1, -1) > c);
    v |= 0x10u * (P(-1, 0) > c);
    v |= 0x08u * (P(1, 0) > c);
    v |= 0x04u * (P(-1, 1) > c);
    v |= 0x02u * (P(0, 1) > c);
    v |= 0x01u * (P(1, 1) > c);
    out[(size_t)y * out_pitch + x] = uint8_t(v);
}

// Natural layout (dst row pitch in elements) or, with planar = 1, the
// matcher's pair-planar scratch layout (pitch ignored).
int launch9x7(const ct_image* src, uint64_t* dst, size_t dst_pitch_elems, int32_t* status, cudaStream_t s,
              int planar) {
    CUtensorMap tm;
    if (int rc = make_tmap_2d(&tm, src->ptr, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, src->width, src->height,
                              src->pitch_bytes, kBoxW, kBoxH))
        return rc;
    dim3 grid((src->width + kTX - 1) / kTX, (src->height + kTY - 1) / kTY);
    census9x7_kernel<<<grid, kNT, 0, s>>>(tm, src->width, src->height, dst, dst_pitch_elems, status, planar);
    CT_LAUNCH_CHECK();
    return CT_OK;
}

// Both views (same size) in one launch.
int launch9x7_pair(const ct_image* a, const ct_image* b, uint64_t* da, uint64_t* db, size_t dst_pitch_elems,
                   int32_t* status, cudaStream_t s, int planar) {
    CUtensorMap ta, tb;
    if (int rc = make_tmap_2d(&ta, a->ptr, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, a->width, a->height, a->pitch_bytes,
                              kBoxW, kBoxH))
        return rc;
    if (int rc = make_tmap_2d(&tb, b->ptr, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, b->width, b->height, b->pitch_bytes,
                              kBoxW, kBoxH))
        return rc;
    dim3 grid((a->width + kTX - 1) / kTX, (a->height + kTY - 1) / kTY, 2);
    census9x7_pair_kernel<<<grid, kNT, 0, s>>>(ta, tb, a->width, a->height, da, db, dst_pitch_elems, status, planar);
    CT_LAUNCH_CHECK();
    return CT_OK;
}

}  // namespace census

// Natural-layout descriptors (row pitch in elements) -> pair-planar scratch.
__global__ void to_planar_kernel(const uint64_t* src, size_t src_pitch, uint64_t* dst, int W, int H) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x < W && y < H) dst[cm::planar_index(x, y, W)] = src[(size_t)y * src_pitch + x];
}

// ---------------------------------------------------------------------------
// CensusTransform::CDriver
// ---------------------------------------------------------------------------
struct CensusHandle : ct_handle {
    CensusHandle() : ct_handle(Kind::Census) {}
    ct_format fmt{};
    ct_census_params par{};
};

// ---------------------------------------------------------------------------
// Census block matcher
// ---------------------------------------------------------------------------
struct BmCensusHandle : ct_handle {
    BmCensusHandle() : ct_handle(Kind::BmCensus) {}
    ~BmCensusHandle() override {
        if (device >= 0) cudaSetDevice(device);
        cudaFree(desc);
        cudaFree(keys);
        cudaFree(counters);
        cudaFree(tmp_lr);
        cudaFree(tmp_rl);
        cudaFree(rl_keys);
    }
    ct_format fmt{};
    ct_census_match_params par{};
    uint64_t* desc = nullptr;      // [2][H][pitch] census descriptors of left, right
    size_t desc_pitch = 0;         // elements
    uint32_t* keys = nullptr;      // ceil(D/64) planes of W*H merge keys
    uint32_t* counters = nullptr;  // one per (strip, column tile); 0 between calls
    uint32_t* rl_keys = nullptr;   // right-view keys of the fused pass, rows of cm::rl_pitch_words(W)
    int rl_next_tag = cm::kRLTags - 1;  // tag of the next fused pass; < 0: reset the plane first
    int fuse_rl = 1;               // process_lr: right-to-left winners from the left-to-right pass
    uint16_t* tmp_lr = nullptr;    // U16 maps for process_lr when the caller wants only one
    uint16_t* tmp_rl = nullptr;
    size_t tmp_pitch = 0;
    CUtensorMap tm_lb, tm_rb, tm_lm, tm_rm;  // left/right as base (box 128) / match (box 192)
    int th = 36;   // strip height, chosen in configure or by the autotuner
    int dpw = 4;   // disparities per warp (kernel variant)
    uint64_t* left_desc() const { return desc; }
    uint64_t* right_desc() const { return desc + (size_t)fmt.height * desc_pitch; }
};

int crosscheck_launch(const ct_image* result, const ct_image* base, const ct_image* other, int tol, int lr,
                      int frame, int32_t* range, cudaStream_t s);  // crosscheck.cu

namespace {

template <typename H>
H* as(ct_handle* h, Kind k) {
    return (h && h->kind == k) ? static_cast<H*>(h) : nullptr;
}

// rl_tag >= 0: the left-to-right pass also bids for the right view into
// h->rl_keys with that tag (the fused kernel).
int census_match_pass_maps(BmCensusHandle* h, int dir, const ct_image* disp, const CUtensorMap& tb,
                           const CUtensorMap& tm, cudaStream_t s, const ct_curves* curves = nullptr,
                           int rl_tag = -1) {
    using namespace cm;
    MatchArgs a{};
    a.W = h->fmt.width; a.H = h->fmt.height;
    // an odd minimum disparity runs as the even one below it with relative
    // d = 0 excluded (see MatchArgs)
    a.dmin = h->par.disp_min & ~1;
    a.dfirst = h->par.disp_min & 1;
    a.D = h->par.disp_count + a.dfirst;
    a.th = h->th;
    a.keys = h->keys;
    a.counters = h->counters;
    a.merge_last = 1;
    a.out = disp->ptr; a.out_pitch = disp->pitch_bytes; a.out_type = disp->type;
    a.status = h->d_status;
    if (curves) {
        a.curve = static_cast<uint32_t*>(curves->ptr);
        a.curve_pitch = curves->pitch_bytes / 4;
        a.curve_groups = (a.D + 3) / 4;
    }
    if (rl_tag >= 0) {  // left-to-right pass bidding for the right view too
        a.rl_keys = h->rl_keys;
        a.rl_pitch = rl_pitch_words(a.W);
        a.rl_tag = uint32_t(rl_tag) << kRLTagShift;
    }
    const cudaError_t e = dir == 0 ? launch_census_match<0>(tb, tm, a, s, h->dpw)
                                   : launch_census_match<1>(tb, tm, a, s, h->dpw);
    if (e != cudaSuccess) return fail(CT_ECUDA, "census match launch failed: %s", cudaGetErrorString(e));
    return CT_OK;
}

// process_lr in one matching pass: the left-to-right kernel decides both
// directions' winners (the left map into lr, the right view's as tagged keys),
// then one kernel writes the right-view map (disp_rl, when asked for) and the
// cross-check of lr against the keys (disp_checked, when asked for).
int census_process_fused(BmCensusHandle* h, const ct_image* lr, const ct_image* disp_rl,
                         const ct_image* disp_checked, int tol, cudaStream_t s) {
    using namespace cm;
    const int W = h->fmt.width, H = h->fmt.height;
    const size_t kpitch = rl_pitch_words(W);
    if (h->rl_next_tag < 0) {  // every tag used since the plane was last set: set it again
        CT_CUDA_TRY(cudaMemsetAsync(h->rl_keys, 0xFF, kpitch * H * 4, s));
        h->rl_next_tag = kRLTags - 1;
    }
    const int tag_no = h->rl_next_tag--;
    if (int rc = census_match_pass_maps(h, 0, lr, h->tm_lb, h->tm_rm, s, nullptr, tag_no)) return rc;
    const uint32_t tag = uint32_t(tag_no) << kRLTagShift;
    const int type = lr->type;
    const int px = 16 / int(pix_size(type));
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((W + 128 * px - 1) / (128 * px), H);
    cfg.blockDim = dim3(128);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void* rl_ptr = disp_rl ? disp_rl->ptr : nullptr;
    const size_t rl_pb = disp_rl ? disp_rl->pitch_bytes : 0;
    void* ck_ptr = disp_checked ? disp_checked->ptr : nullptr;
    const size_t ck_pb = disp_checked ? disp_checked->pitch_bytes : 0;
    if (type == CT_PIX_U8)
        CT_CUDA_TRY(cudaLaunchKernelEx(&cfg, rl_check_kernel<uint8_t>, h->rl_keys, kpitch, tag, W, H, int(kAR),
                                       static_cast<uint8_t*>(rl_ptr), rl_pb, static_cast<const uint8_t*>(lr->ptr),
                                       lr->pitch_bytes, static_cast<uint8_t*>(ck_ptr), ck_pb, tol));
    else
        CT_CUDA_TRY(cudaLaunchKernelEx(&cfg, rl_check_kernel<uint16_t>, h->rl_keys, kpitch, tag, W, H, int(kAR),
                                       static_cast<uint16_t*>(rl_ptr), rl_pb, static_cast<const uint16_t*>(lr->ptr),
                                       lr->pitch_bytes, static_cast<uint16_t*>(ck_ptr), ck_pb, tol));
    CT_LAUNCH_CHECK();
    return CT_OK;
}

int census_match_pass(BmCensusHandle* h, int dir, const ct_image* disp, cudaStream_t s,
                      const ct_curves* curves = nullptr) {
    return dir == 0 ? census_match_pass_maps(h, 0, disp, h->tm_lb, h->tm_rm, s, curves)
                    : census_match_pass_maps(h, 1, disp, h->tm_rb, h->tm_lm, s, curves);
}

int census_both(BmCensusHandle* h, const ct_image* left, const ct_image* right, cudaStream_t s) {
    return census::launch9x7_pair(left, right, h->left_desc(), h->right_desc(), h->desc_pitch, h->d_status, s, 1);
}

}  // namespace

}  // namespace ct

using namespace ct;

extern "C" {

int ct_census_create(ct_handle** out) {
    clear_error();
    if (!out) return fail(CT_EINVAL, "null output handle pointer");
    *out = new CensusHandle();
    return CT_OK;
}

int ct_census_configure(ct_handle* hh, int32_t device, const ct_format* fmt, const ct_census_params* p) {
    clear_error();
    auto* h = as<CensusHandle>(hh, Kind::Census);
    if (!h) return fail(CT_ESTATE, "not a census handle");
    if (!fmt || !p) return fail(CT_EINVAL, "null format or parameters");
    if (fmt->type != CT_PIX_U8) return fail(CT_ETYPE, "census input must be U8 (TPixel_Lum_UInt8)");
    if (fmt->width < 1 || fmt->height < 1) return fail(CT_EINVAL, "bad size");
    if (p->window != CT_CENSUS_9X7 && p->window != CT_CENSUS_3X3) return fail(CT_EINVAL, "unknown census window");
    if (int rc = use_device(device)) return rc;
    h->device = device;
    if (int rc = h->init_status()) return rc;
    h->fmt = *fmt;
    h->par = *p;
    h->configured = true;
    return CT_OK;
}

int ct_census_process_pair(ct_handle* hh, const ct_image* dst_left, const ct_image* dst_right,
                           const ct_image* src_left, const ct_image* src_right, ct_stream stream) {
    clear_error();
    auto* h = as<CensusHandle>(hh, Kind::Census);
    if (!h) return fail(CT_ESTATE, "not a census handle");
    if (!h->configured) return fail(CT_ESTATE, "process before configure");
    if (h->par.window != CT_CENSUS_9X7) return fail(CT_EINVAL, "the pair launch is built for the 9x7 transform");
    for (const ct_image* im : {src_left, src_right})
        if (int rc = check_image(im, "src", 1u << CT_PIX_U8)) return rc;
    for (const ct_image* im : {dst_left, dst_right})
        if (int rc = check_image(im, "dst", 1u << CT_PIX_U64)) return rc;
    for (const ct_image* im : {dst_left, dst_right, src_right})
        if (int rc = check_same_size(im, src_left, "image", "src_left")) return rc;
    if (src_left->width != h->fmt.width || src_left->height != h->fmt.height)
        return fail(CT_EFORMAT, "image size differs from the configured format");
    if (dst_left->pitch_bytes != dst_right->pitch_bytes) return fail(CT_EFORMAT, "the two outputs need one pitch");
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    return census::launch9x7_pair(src_left, src_right, static_cast<uint64_t*>(dst_left->ptr),
                                  static_cast<uint64_t*>(dst_right->ptr), dst_left->pitch_bytes / 8, h->d_status, s, 0);
}

int ct_census_process(ct_handle* hh, const ct_image* dst, const ct_image* src, ct_stream stream) {
    clear_error();
    auto* h = as<CensusHandle>(hh, Kind::Census);
    if (!h) return fail(CT_ESTATE, "not a census handle");
    if (!h->configured) return fail(CT_ESTATE, "process before configure");
    if (int rc = check_image(src, "src", 1u << CT_PIX_U8)) return rc;
    const uint32_t dt = h->par.window == CT_CENSUS_9X7 ? (1u << CT_PIX_U64) : (1u << CT_PIX_U8);
    if (int rc = check_image(dst, "dst", dt)) return rc;
    if (int rc = check_same_size(dst, src, "dst", "src")) return rc;
    if (src->width != h->fmt.width || src->height != h->fmt.height)
        return fail(CT_EFORMAT, "image size differs from the configured format");
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    if (h->par.window == CT_CENSUS_9X7) {
        return census::launch9x7(src, static_cast<uint64_t*>(dst->ptr), dst->pitch_bytes / 8, h->d_status, s, 0);
    }
    dim3 blk(32, 8), grid((src->width + 31) / 32, (src->height + 7) / 8);
    census::census3x3_kernel<<<grid, blk, 0, s>>>(static_cast<const uint8_t*>(src->ptr), src->pitch_bytes,
                                                  src->width, src->height, static_cast<uint8_t*>(dst->ptr),
                                                  dst->pitch_bytes);
    CT_LAUNCH_CHECK();
    return CT_OK;
}

int ct_bm_census_create(ct_handle** out) {
    clear_error();
    if (!out) return fail(CT_EINVAL, "null output handle pointer");
    *out = new BmCensusHandle();
    return CT_OK;
}

int ct_bm_census_configure(ct_handle* hh, int32_t device, const ct_format* fmt, const ct_census_match_params* p) {
    clear_error();
    auto* h = as<BmCensusHandle>(hh, Kind::BmCensus);
    if (!h) return fail(CT_ESTATE, "not a census matcher handle");
    if (!fmt || !p) return fail(CT_EINVAL, "null format or parameters");
    if (fmt->type != CT_PIX_U8) return fail(CT_ETYPE, "matcher input must be U8 (TPixel_Lum_UInt8)");
    if (fmt->width < 8 || fmt->height < 8 || fmt->width > 32768 || fmt->height > 32768)
        return fail(CT_EINVAL, "image size %dx%d out of range (8..32768)", fmt->width, fmt->height);
    if (p->disp_count < 1 || p->disp_count > 256) return fail(CT_EINVAL, "disp_count must be 1..256");
    if (p->agg_radius != cm::kAR) return fail(CT_EINVAL, "only agg_radius 2 (5x5) is built");
    if (p->disp_min < 0 || p->disp_min + p->disp_count > 0xFFEF)
        return fail(CT_EINVAL, "disp_min must be >= 0 with disp_min + disp_count <= 65519");
    if (int rc = use_device(device)) return rc;
    // release a previous configuration
    cudaFree(h->desc); cudaFree(h->keys); cudaFree(h->counters); cudaFree(h->tmp_lr); cudaFree(h->tmp_rl);
    cudaFree(h->rl_keys);
    h->desc = nullptr; h->keys = nullptr; h->counters = nullptr; h->tmp_lr = nullptr; h->tmp_rl = nullptr;
    h->rl_keys = nullptr;
    h->device = device;
    if (int rc = h->init_status()) return rc;
    const int W = fmt->width, H = fmt->height;
    h->desc_pitch = cm::planar_pitch(W);  // pair-planar layout
    if (cudaMalloc(&h->desc, 2 * h->desc_pitch * H * 8) != cudaSuccess) return fail(CT_ENOMEM, "descriptor scratch");
    const size_t zplanes = (p->disp_count + (p->disp_min & 1) + cm::kDPC - 1) / cm::kDPC;
    if (cudaMalloc(&h->keys, zplanes * W * H * 4) != cudaSuccess) return fail(CT_ENOMEM, "key scratch");
    // counters for the shortest strips any launch shape uses (11 rows)
    const size_t ngroups = size_t((H + 10) / 11) * ((W + cm::kTWO - 1) / cm::kTWO);
    if (cudaMalloc(&h->counters, ngroups * 4) != cudaSuccess) return fail(CT_ENOMEM, "counter scratch");
    CT_CUDA_TRY(cudaMemset(h->counters, 0, ngroups * 4));
    h->tmp_pitch = ((size_t)W * 2 + 255) / 256 * 256;
    if (cudaMalloc(&h->tmp_lr, h->tmp_pitch * H) != cudaSuccess) return fail(CT_ENOMEM, "map scratch");
    if (cudaMalloc(&h->tmp_rl, h->tmp_pitch * H) != cudaSuccess) return fail(CT_ENOMEM, "map scratch");
    const size_t rl_bytes = cm::rl_pitch_words(W) * H * 4;
    if (cudaMalloc(&h->rl_keys, rl_bytes) != cudaSuccess) return fail(CT_ENOMEM, "right-view key scratch");
    CT_CUDA_TRY(cudaMemset(h->rl_keys, 0xFF, rl_bytes));
    h->rl_next_tag = cm::kRLTags - 1;
    h->fmt = *fmt;  // left_desc() / right_desc() below depend on the height
    h->th = cm::pick_strip_height(W, H, p->disp_count, sm_count(device));
    CT_CUDA_TRY(cm::prepare_census_match());
    h->par = *p;
    using namespace cm;
    if (int rc = make_planar_maps(&h->tm_lb, &h->tm_rm, h->left_desc(), h->right_desc(), W, H)) return rc;
    if (int rc = make_planar_maps(&h->tm_rb, &h->tm_lm, h->right_desc(), h->left_desc(), W, H)) return rc;
    h->configured = true;
    return CT_OK;
}

static int check_match_io(BmCensusHandle* h, const ct_image* left, const ct_image* right) {
    if (!h->configured) return fail(CT_ESTATE, "process before configure");
    if (int rc = check_image(left, "left", 1u << CT_PIX_U8)) return rc;
    if (int rc = check_image(right, "right", 1u << CT_PIX_U8)) return rc;
    if (int rc = check_same_size(left, right, "left", "right")) return rc;
    if (left->width != h->fmt.width || left->height != h->fmt.height)
        return fail(CT_EFORMAT, "image size differs from the configured format");
    return CT_OK;
}

static int check_disp_out(BmCensusHandle* h, const ct_image* d, const char* name) {
    if (int rc = check_image(d, name, (1u << CT_PIX_U8) | (1u << CT_PIX_U16))) return rc;
    if (d->width != h->fmt.width || d->height != h->fmt.height)
        return fail(CT_EFORMAT, "%s size differs from the configured format", name);
    if (d->type == CT_PIX_U8 && h->par.disp_min + h->par.disp_count > 255)
        return fail(CT_ETYPE, "U8 maps need disp_min + disp_count <= 255");
    return CT_OK;
}

int ct_bm_census_process(ct_handle* hh, const ct_image* disp, const ct_image* left, const ct_image* right,
                         ct_stream stream) {
    clear_error();
    auto* h = as<BmCensusHandle>(hh, Kind::BmCensus);
    if (!h) return fail(CT_ESTATE, "not a census matcher handle");
    if (int rc = check_match_io(h, left, right)) return rc;
    if (int rc = check_disp_out(h, disp, "disp")) return rc;
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    if (int rc = census_both(h, left, right, s)) return rc;
    return census_match_pass(h, h->par.left_to_right ? 0 : 1, disp, s);
}

int ct_curves_pitch(int32_t width, size_t* pitch_bytes) {
    clear_error();
    if (!pitch_bytes || width < 1) return fail(CT_EINVAL, "bad width or null output");
    *pitch_bytes = cm::curve_pitch_words(width) * 4;
    return CT_OK;
}

int ct_bm_census_process_curves(ct_handle* hh, const ct_image* disp, const ct_curves* curves,
                                const ct_image* left, const ct_image* right, ct_stream stream) {
    clear_error();
    auto* h = as<BmCensusHandle>(hh, Kind::BmCensus);
    if (!h) return fail(CT_ESTATE, "not a census matcher handle");
    if (int rc = check_match_io(h, left, right)) return rc;
    if (int rc = check_disp_out(h, disp, "disp")) return rc;
    if (!curves || !curves->ptr) return fail(CT_EINVAL, "null curve volume");
    if (h->par.disp_min != 0) return fail(CT_EINVAL, "cost curves are built for disp_min 0");
    if (curves->width != h->fmt.width || curves->height != h->fmt.height ||
        curves->disp_count != h->par.disp_count)
        return fail(CT_EFORMAT, "curve volume size differs from the configured format");
    if (reinterpret_cast<uintptr_t>(curves->ptr) % 16 || curves->pitch_bytes % 16 ||
        curves->pitch_bytes < 4 * (size_t(h->fmt.width) + 2))
        return fail(CT_EINVAL, "curve volume needs a 16-byte aligned pointer and pitch >= 4 * (width + 2)");
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    if (int rc = census_both(h, left, right, s)) return rc;
    return census_match_pass(h, h->par.left_to_right ? 0 : 1, disp, s, curves);
}

int ct_bm_census_process_lr(ct_handle* hh, const ct_image* disp_lr, const ct_image* disp_rl,
                            const ct_image* disp_checked, int32_t tol, const ct_image* left,
                            const ct_image* right, ct_stream stream) {
    clear_error();
    auto* h = as<BmCensusHandle>(hh, Kind::BmCensus);
    if (!h) return fail(CT_ESTATE, "not a census matcher handle");
    if (int rc = check_match_io(h, left, right)) return rc;
    if (!disp_lr && !disp_rl && !disp_checked) return fail(CT_EINVAL, "no output requested");
    if (tol < 0) return fail(CT_EINVAL, "tol must be >= 0");
    int32_t t = -1;
    for (const ct_image* d : {disp_lr, disp_rl, disp_checked}) {
        if (!d) continue;
        if (int rc = check_disp_out(h, d, "disp")) return rc;
        if (t >= 0 && d->type != t) return fail(CT_ETYPE, "all output maps must have the same type");
        t = d->type;
    }
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    if (int rc = census_both(h, left, right, s)) return rc;
    const int W = h->fmt.width, H = h->fmt.height;
    ct_image tlr{h->tmp_lr, h->tmp_pitch, W, H, t, 0};
    ct_image trl{h->tmp_rl, h->tmp_pitch, W, H, t, 0};
    if (t == CT_PIX_U8) { tlr.pitch_bytes = trl.pitch_bytes = h->tmp_pitch; }
    const ct_image* lr = disp_lr ? disp_lr : &tlr;
    const ct_image* rl = disp_rl ? disp_rl : &trl;
    const bool need_lr = disp_lr || disp_checked, need_rl = disp_rl || disp_checked;
    if (need_lr && need_rl && h->fuse_rl)  // the same maps as two passes
        return census_process_fused(h, lr, disp_rl, disp_checked, tol, s);
    {
        if (need_lr)
            if (int rc = census_match_pass(h, 0, lr, s)) return rc;
        if (need_rl)
            if (int rc = census_match_pass(h, 1, rl, s)) return rc;
    }
    if (disp_checked) return crosscheck_launch(disp_checked, lr, rl, tol, 1, /*frame*/ 0, nullptr, s);
    return CT_OK;
}

int ct_bm_census_autotune(ct_handle* hh, const ct_image* left, const ct_image* right, ct_stream stream) {
    clear_error();
    auto* h = as<BmCensusHandle>(hh, Kind::BmCensus);
    if (!h) return fail(CT_ESTATE, "not a census matcher handle");
    if (int rc = check_match_io(h, left, right)) return rc;
    if (int rc = use_device(h->device)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    if (int rc = census_both(h, left, right, s)) return rc;
    const int W = h->fmt.width, H = h->fmt.height, D = h->par.disp_count;
    const int dir = h->par.left_to_right ? 0 : 1;
    // candidates: both variants x the model's strip height and its neighbours
    const int th0 = cm::pick_strip_height(W, H, D, sm_count(h->device));
    int ths[6] = {th0, th0 - 10, th0 + 10, th0 - 40, 36, 61};
    ct_image out{h->tmp_lr, h->tmp_pitch, W, H, CT_PIX_U16, 0};
    cudaEvent_t e0, e1;
    CT_CUDA_TRY(cudaEventCreate(&e0));
    CT_CUDA_TRY(cudaEventCreate(&e1));
    float best_ms = 1e30f;
    int best_th = th0, best_dpw = 4;
    int rc = CT_OK;
    for (int dpw : {4, 8}) {
        for (int th : ths) {
            if (th < 11 || (th + 2 * cm::kAR) % cm::kRB != 0) continue;
            h->dpw = dpw;
            h->th = th;
            if ((rc = census_match_pass(h, dir, &out, s))) break;  // warm-up
            float t = 1e30f;
            for (int rep = 0; rep < 3 && rc == CT_OK; ++rep) {
                cudaEventRecord(e0, s);
                rc = census_match_pass(h, dir, &out, s);
                cudaEventRecord(e1, s);
                const cudaError_t e = cudaEventSynchronize(e1);
                if (e != cudaSuccess) { rc = fail(CT_ECUDA, "autotune timing failed: %s", cudaGetErrorString(e)); break; }
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                t = ms < t ? ms : t;
            }
            if (rc) break;
            if (t < best_ms) { best_ms = t; best_th = th; best_dpw = dpw; }
        }
        if (rc) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h->th = best_th;
    h->dpw = best_dpw;
    return rc;
}

int ct_bm_census_tuning(ct_handle* hh, int32_t* strip_height, int32_t* disp_per_warp) {
    clear_error();
    auto* h = as<BmCensusHandle>(hh, Kind::BmCensus);
    if (!h) return fail(CT_ESTATE, "not a census matcher handle");
    if (!h->configured) return fail(CT_ESTATE, "tuning before configure");
    if (strip_height) *strip_height = h->th;
    if (disp_per_warp) *disp_per_warp = h->dpw;
    return CT_OK;
}

int ct_bm_census_set_fused_lr(ct_handle* hh, int32_t enable) {
    clear_error();
    auto* h = as<BmCensusHandle>(hh, Kind::BmCensus);
    if (!h) return fail(CT_ESTATE, "not a census matcher handle");
    if (enable != 0 && enable != 1) return fail(CT_EINVAL, "enable must be 0 or 1");
    h->fuse_rl = enable;
    return CT_OK;
}

int ct_bm_census_set_tuning(ct_handle* hh, int32_t strip_height, int32_t disp_per_warp) {
    clear_error();
    auto* h = as<BmCensusHandle>(hh, Kind::BmCensus);
    if (!h) return fail(CT_ESTATE, "not a census matcher handle");
    if (strip_height < 11 || strip_height > 511 || (strip_height + 2 * cm::kAR) % cm::kRB != 0)
        return fail(CT_EINVAL, "strip_height must be 11..511 with strip_height + 4 a multiple of 5");
    if (disp_per_warp != 4 && disp_per_warp != 8) return fail(CT_EINVAL, "disp_per_warp must be 4 or 8");
    h->th = strip_height;
    h->dpw = disp_per_warp;
    return CT_OK;
}

int ct_bm_census_match_desc(ct_handle* hh, const ct_image* disp, const ct_image* desc_base,
                            const ct_image* desc_match, int32_t left_to_right, ct_stream stream) {
    clear_error();
    auto* h = as<BmCensusHandle>(hh, Kind::BmCensus);
    if (!h) return fail(CT_ESTATE, "not a census matcher handle");
    if (!h->configured) return fail(CT_ESTATE, "process before configure");
    if (int rc = check_image(desc_base, "desc_base", 1u << CT_PIX_U64)) return rc;
    if (int rc = check_image(desc_match, "desc_match", 1u << CT_PIX_U64)) return rc;
    if (int rc = check_same_size(desc_base, desc_match, "desc_base", "desc_match")) return rc;
    if (desc_base->width != h->fmt.width || desc_base->height != h->fmt.height)
        return fail(CT_EFORMAT, "descriptor size differs from the configured format");
    if (int rc = check_disp_out(h, disp, "disp")) return rc;
    if (int rc = use_device(h->device)) return rc;
    const int W = h->fmt.width, H = h->fmt.height;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    h->last_stream = s;
    // the caller's natural-layout descriptors -> the handle's pair-planar scratch
    const int dir = left_to_right ? 0 : 1;
    uint64_t* base_dst = dir == 0 ? h->left_desc() : h->right_desc();
    uint64_t* match_dst = dir == 0 ? h->right_desc() : h->left_desc();
    dim3 cb(256), cg((W + 255) / 256, H);
    to_planar_kernel<<<cg, cb, 0, s>>>(static_cast<const uint64_t*>(desc_base->ptr), desc_base->pitch_bytes / 8,
                                       base_dst, W, H);
    to_planar_kernel<<<cg, cb, 0, s>>>(static_cast<const uint64_t*>(desc_match->ptr), desc_match->pitch_bytes / 8,
                                       match_dst, W, H);
    CT_LAUNCH_CHECK();
    return census_match_pass(h, dir, disp, s);
}

}  // extern "C"
