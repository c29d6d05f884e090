// stream.cpp — streamed census stereo (ct_census_stream_*): frames in host
// memory in, cross-checked disparity maps in host memory out. Three device
// slots rotate over three streams:
//
//   up    waits until its slot's previous frame has been matched, copies the
//         left and right images in, records `uploaded`;
//   run   waits for `uploaded` and for the slot's previous map to be copied
//         out, runs ct_bm_census_process_lr into the slot's map, records
//         `computed`;
//   down  waits for `computed`, copies the map out, records `downloaded`.
//
// So the upload of frame k + 1 and the download of frame k - 1 run on the copy
// engines while frame k is matched; nothing on the host waits unless the
// caller asks (ct_census_stream_wait).
#include "ct_internal.h"

namespace ct {
namespace {

constexpr int kSlots = 3;

struct StreamHandle : ct_handle {
    StreamHandle() : ct_handle(Kind::Stream) {}
    ~StreamHandle() override { release(); }

    struct Slot {
        void* L = nullptr;
        void* R = nullptr;
        void* out = nullptr;
        cudaEvent_t uploaded = nullptr, computed = nullptr, downloaded = nullptr;
    };

    ct_handle* matcher = nullptr;  // the census matcher doing the work (owned)
    int W = 0, H = 0, tol = 1, out_type = CT_PIX_U8;
    size_t in_pitch = 0, out_pitch = 0;
    cudaStream_t up = nullptr, run = nullptr, down = nullptr;
    Slot slot[kSlots];
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    bool mark_pending = false, marked = false;
    int64_t submitted = 0;

    void release() {
        if (device >= 0) cudaSetDevice(device);
        for (cudaStream_t s : {up, run, down})
            if (s) cudaStreamSynchronize(s);
        for (Slot& s : slot) {
            for (cudaEvent_t e : {s.uploaded, s.computed, s.downloaded})
                if (e) cudaEventDestroy(e);
            for (void* p : {s.L, s.R, s.out})
                if (p) cudaFree(p);
            s = Slot{};
        }
        for (cudaEvent_t e : {t0, t1})
            if (e) cudaEventDestroy(e);
        for (cudaStream_t s : {up, run, down})
            if (s) cudaStreamDestroy(s);
        up = run = down = nullptr;
        t0 = t1 = nullptr;
        // the status word belongs to the matcher; do not let ~Handle free it
        d_status = nullptr;
        last_stream = nullptr;
        ct_destroy(matcher);
        matcher = nullptr;
        configured = false;
        submitted = 0;
        mark_pending = marked = false;
    }
};

StreamHandle* as_stream(ct_handle* h) {
    return (h && h->kind == Kind::Stream) ? static_cast<StreamHandle*>(h) : nullptr;
}

}  // namespace
}  // namespace ct

using namespace ct;

extern "C" {

int ct_census_stream_create(ct_handle** out) {
    clear_error();
    if (!out) return fail(CT_EINVAL, "null output handle pointer");
    *out = new StreamHandle();
    return CT_OK;
}

int ct_census_stream_configure(ct_handle* hh, int32_t device, const ct_format* fmt, const ct_census_match_params* p,
                               int32_t tol, int32_t out_type) {
    clear_error();
    auto* h = as_stream(hh);
    if (!h) return fail(CT_ESTATE, "not a census stream handle");
    if (!fmt || !p) return fail(CT_EINVAL, "null format or parameters");
    if (tol < 0) return fail(CT_EINVAL, "tol must be >= 0");
    if (out_type != CT_PIX_U8 && out_type != CT_PIX_U16) return fail(CT_ETYPE, "maps must be U8 or U16");
    if (out_type == CT_PIX_U8 && p->disp_min + p->disp_count > 255)
        return fail(CT_ETYPE, "U8 maps hold disparities below 255 (disp_min + disp_count <= 255)");
    h->release();
    if (int rc = ct_bm_census_create(&h->matcher)) return rc;
    if (int rc = ct_bm_census_configure(h->matcher, device, fmt, p)) return rc;
    if (int rc = use_device(device)) return rc;
    h->device = device;
    h->W = fmt->width;
    h->H = fmt->height;
    h->tol = tol;
    h->out_type = out_type;
    for (cudaStream_t* s : {&h->up, &h->run, &h->down}) CT_CUDA_TRY(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking));
    for (auto& s : h->slot) {
        for (cudaEvent_t* e : {&s.uploaded, &s.computed, &s.downloaded})
            CT_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        size_t pl = 0, pr = 0, po = 0;
        if (cudaMallocPitch(&s.L, &pl, size_t(h->W), size_t(h->H)) != cudaSuccess ||
            cudaMallocPitch(&s.R, &pr, size_t(h->W), size_t(h->H)) != cudaSuccess ||
            cudaMallocPitch(&s.out, &po, size_t(h->W) * pix_size(out_type), size_t(h->H)) != cudaSuccess)
            return fail(CT_ENOMEM, "stream slot images");
        h->in_pitch = pl;
        h->out_pitch = po;
    }
    CT_CUDA_TRY(cudaEventCreate(&h->t0));
    CT_CUDA_TRY(cudaEventCreate(&h->t1));
    // device status: the matcher's word, read after its (run) stream
    h->d_status = h->matcher->d_status;
    h->last_stream = h->run;
    h->configured = true;
    return CT_OK;
}

int ct_census_stream_submit(ct_handle* hh, const void* left, size_t left_pitch, const void* right,
                            size_t right_pitch, void* checked, size_t checked_pitch, int64_t* frame) {
    clear_error();
    auto* h = as_stream(hh);
    if (!h || !h->configured) return fail(CT_ESTATE, "not a configured census stream handle");
    if (!left || !right || !checked) return fail(CT_EINVAL, "null image");
    const size_t row_out = size_t(h->W) * pix_size(h->out_type);
    if (left_pitch < size_t(h->W) || right_pitch < size_t(h->W) || checked_pitch < row_out)
        return fail(CT_EINVAL, "host pitch smaller than a row");
    if (int rc = use_device(h->device)) return rc;
    const int64_t k = h->submitted;
    auto& s = h->slot[k % kSlots];
    const size_t W = size_t(h->W), H = size_t(h->H);
    // up: the slot's images are free once its previous frame has been matched
    CT_CUDA_TRY(cudaStreamWaitEvent(h->up, s.computed, 0));
    if (h->mark_pending) {
        CT_CUDA_TRY(cudaEventRecord(h->t0, h->up));
        h->mark_pending = false;
        h->marked = true;
    }
    CT_CUDA_TRY(cudaMemcpy2DAsync(s.L, h->in_pitch, left, left_pitch, W, H, cudaMemcpyHostToDevice, h->up));
    CT_CUDA_TRY(cudaMemcpy2DAsync(s.R, h->in_pitch, right, right_pitch, W, H, cudaMemcpyHostToDevice, h->up));
    CT_CUDA_TRY(cudaEventRecord(s.uploaded, h->up));
    // run: inputs present, and the slot's previous map copied out
    CT_CUDA_TRY(cudaStreamWaitEvent(h->run, s.uploaded, 0));
    CT_CUDA_TRY(cudaStreamWaitEvent(h->run, s.downloaded, 0));
    const ct_image L{s.L, h->in_pitch, h->W, h->H, CT_PIX_U8, 0};
    const ct_image R{s.R, h->in_pitch, h->W, h->H, CT_PIX_U8, 0};
    const ct_image O{s.out, h->out_pitch, h->W, h->H, h->out_type, 0};
    if (int rc = ct_bm_census_process_lr(h->matcher, nullptr, nullptr, &O, h->tol, &L, &R,
                                         reinterpret_cast<ct_stream>(h->run)))
        return rc;
    CT_CUDA_TRY(cudaEventRecord(s.computed, h->run));
    // down
    CT_CUDA_TRY(cudaStreamWaitEvent(h->down, s.computed, 0));
    CT_CUDA_TRY(cudaMemcpy2DAsync(checked, checked_pitch, s.out, h->out_pitch, row_out, H, cudaMemcpyDeviceToHost,
                                  h->down));
    CT_CUDA_TRY(cudaEventRecord(s.downloaded, h->down));
    h->submitted = k + 1;
    if (frame) *frame = k;
    return CT_OK;
}

int ct_census_stream_wait(ct_handle* hh, int64_t frame) {
    clear_error();
    auto* h = as_stream(hh);
    if (!h || !h->configured) return fail(CT_ESTATE, "not a configured census stream handle");
    if (frame < 0 || frame >= h->submitted) return fail(CT_EINVAL, "frame %lld was not submitted", (long long)frame);
    if (int rc = use_device(h->device)) return rc;
    // the slot's event marks this frame or a later one in the same slot;
    // frames leave the down stream in order, so either way this frame is done
    CT_CUDA_TRY(cudaEventSynchronize(h->slot[frame % kSlots].downloaded));
    return CT_OK;
}

int ct_census_stream_timer_start(ct_handle* hh) {
    clear_error();
    auto* h = as_stream(hh);
    if (!h || !h->configured) return fail(CT_ESTATE, "not a configured census stream handle");
    h->mark_pending = true;
    h->marked = false;
    return CT_OK;
}

int ct_census_stream_timer_stop(ct_handle* hh, float* ms) {
    clear_error();
    auto* h = as_stream(hh);
    if (!h || !h->configured) return fail(CT_ESTATE, "not a configured census stream handle");
    if (!ms) return fail(CT_EINVAL, "null output");
    if (!h->marked) return fail(CT_ESTATE, "no frame submitted since ct_census_stream_timer_start");
    if (int rc = use_device(h->device)) return rc;
    CT_CUDA_TRY(cudaEventRecord(h->t1, h->down));
    CT_CUDA_TRY(cudaEventSynchronize(h->t1));
    CT_CUDA_TRY(cudaEventElapsedTime(ms, h->t0, h->t1));
    h->marked = false;
    return CT_OK;
}

}  // extern "C"
