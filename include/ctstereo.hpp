/* ctstereo.hpp — header-only C++ layer over the ctstereo C ABI that keeps the
 * reference's driver shape, so code written against CluTec.Cuda's MultiView
 * drivers switches by changing includes and a namespace:
 *
 *     Clu::Cuda::BlockMatcherNCC::CDriver xMatcher;         // reference
 *     ctstereo::BlockMatcherNCC::CDriver xMatcher;          // this library
 *
 *     xMatcher.Configure(xDevice, xFormat, xPars);
 *     double dMs = ProcessKernel(xMatcher, surfDisp, surfL, surfR, surfNone, surfNone);
 *
 * Mapping (reference file:line -> here):
 *   Clu::Cuda::CDevice, Clu::SImageFormat       -> CDevice, SImageFormat
 *   Clu::Cuda::_CDeviceSurface (DeviceSurface.h:43-264; cudaArray + surface)
 *                                                -> _CDeviceSurface (pitched view)
 *   Clu::Cuda::CDeviceSurface (Create / CopyFrom / CopyInto)
 *                                                -> CDeviceSurface (owning)
 *   Clu::Cuda::CKernelDriverBase (KernelDriverBase.h:46-177), ProcessKernel
 *     (KernelDriverBase.h:180-199)              -> CKernelDriverBase, ProcessKernel
 *   Clu::Cuda::EDisparityId (DisparityId.h:35-47) -> EDisparityId
 *   ColorDisparityImage::{EStyle, SParameter, CDriver} (ColorDisparityImage.h:37-120),
 *     into a headless RGBA8 / U16 device image
 *   CensusTransform::CDriver (CensusTransform.h:44-70)
 *   BlockMatcherSAD1::{EConfig, SParameter, CDriver} (BlockMatcherSAD1.h:42-127)
 *   BlockMatcherNCC::{EConfig, SParameter, CDriver} (BlockMatcherNCC.h:41-144)
 *   BlockMatcherAW1::{EConfig, ESimType, SParameter, CDriver} (BlockMatcherAW1.h:41-157)
 *   CrossCheckDisparityMaps::{SParameter, CDriver} (CrossCheckDisparityMaps.h:38-117)
 * and, with no reference counterpart: BlockMatcherCensus (census pipeline in
 * one call, with cost-curve export), CensusStream (host frames in, maps out,
 * copies overlapping the matching), BatchStereo (many pairs per launch) and
 * ConfidenceNet (learned confidence over the cost curves).
 *
 * Errors: every failing C call becomes a CError exception carrying the CT_E*
 * code and ct_last_error_string(), the role of CLU_EXCEPTION in the
 * reference. The C ABI itself never throws.
 *
 * Differences a caller sees (the build's semantics, not the reference's):
 *   - Disparities run from _SDisparityConfig::iMin (SAD1: iOffset) over
 *     iRange values; U16 disparity maps hold d + EDisparityId::First or an
 *     ID, U8 maps hold d or 255 (iMin + iRange <= 255).
 *   - The output surface's type picks the semantics. EDataType::UInt16x4
 *     gets the reference's own TPixelEx output (ct_bm_compat_*: its score
 *     quantisation, scan order, gates, ID thresholds and specificity
 *     channels; BlockMatcher1, BlockMatcherAW2 and the AW1 2-of-4 patches
 *     write only that, or its x channel into UInt16). UInt8 / UInt16 / Single
 *     get the plain winner-take-all maps (exhaustive search, lowest
 *     disparity on ties, unquantised NCC, gradient gate); the ID thresholds
 *     (fSadThresh, fNccThresh, fSimThresh, iMinDeltaThresh, fMinDeltaThresh)
 *     label the TPixelEx output only and must be 0 on that path.
 *   - Guided matching (iUseDispInput + xImageDispInit) searches per 16 x 16
 *     block (see ct_bm_ncc_process / ct_bm_aw_process_guided).
 *   - BlockMatcherAW1 computes the "best of 5 shifted 7x7 windows" cost with
 *     sub-pixel refinement (EConfig::Shifted5_7x7); the reference's 2-of-4
 *     sub-window configurations throw.
 *   - CrossCheckDisparityMaps::DispMin / DispMax return disparities (d, not
 *     d + First) and synchronise the last Process stream.
 *   - Process is asynchronous on the driver's stream (SetStream; default
 *     stream 0); ProcessKernel records events around it and waits, like the
 *     reference's Begin / End.
 */
#ifndef CTSTEREO_HPP
#define CTSTEREO_HPP

#include "ctstereo.h"

#include <cuda_runtime_api.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace ctstereo {

/* ---- errors --------------------------------------------------------------- */

class CError : public std::runtime_error {
public:
    CError(int code, const std::string& what) : std::runtime_error(what), m_iCode(code) {}
    int Code() const { return m_iCode; }

private:
    int m_iCode;
};

inline void Ensure(int rc, const char* what) {
    if (rc != CT_OK) throw CError(rc, std::string(what) + ": " + ct_last_error_string());
}

inline void EnsureCuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CError(CT_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

/* ---- device, format, disparity IDs ----------------------------------------- */

struct CDevice {
    int iDevice = 0;
    CDevice() = default;
    explicit CDevice(int device) : iDevice(device) {}
};

enum class EDataType : int32_t {
    UInt8 = CT_PIX_U8,
    UInt16 = CT_PIX_U16,
    UInt64 = CT_PIX_U64,
    Single = CT_PIX_F32,
    RGBA8 = CT_PIX_RGBA8,  // 4 bytes: r, g, b, a
    RGBA_Single = CT_PIX_F32X4,  // 4 floats (3D map)
    UInt16x4 = CT_PIX_U16X4,     // 4 x uint16: the reference matchers' TPixelEx output
};

inline size_t BytesPerPixel(EDataType t) {
    switch (t) {
        case EDataType::UInt8: return 1;
        case EDataType::UInt16: return 2;
        case EDataType::UInt64: return 8;
        case EDataType::Single: return 4;
        case EDataType::RGBA8: return 4;
        case EDataType::RGBA_Single: return 16;
        case EDataType::UInt16x4: return 8;
    }
    return 0;
}

/* Luminance images only: the matchers take one channel (the reference
 * requires TPixel_Lum_UInt8 inputs, BlockMatcherNCC.cu:1411-1419). */
struct SImageFormat {
    int iWidth = 0;
    int iHeight = 0;
    EDataType eDataType = EDataType::UInt8;

    SImageFormat() = default;
    SImageFormat(int w, int h, EDataType t = EDataType::UInt8) : iWidth(w), iHeight(h), eDataType(t) {}
    bool operator==(const SImageFormat& o) const {
        return iWidth == o.iWidth && iHeight == o.iHeight && eDataType == o.eDataType;
    }
    ct_format ToC() const { return ct_format{iWidth, iHeight, static_cast<int32_t>(eDataType)}; }
};

enum class EDisparityId : uint16_t {
    First = CT_DISP_FIRST,
    Last = CT_DISP_LAST,
    Unknown = CT_DISP_UNKNOWN,
    CannotEvaluate = CT_DISP_CANNOT_EVALUATE,
    Saturated = CT_DISP_SATURATED,
    NotFound = CT_DISP_NOT_FOUND,
    NotSpecific = CT_DISP_NOT_SPECIFIC,
    NotUnique = CT_DISP_NOT_UNIQUE,
    Inconsistent = CT_DISP_INCONSISTENT,
};

/* Replaces _SDisparityConfig (CluTec.ImgProc/DisparityConfig.h, not in the
 * reference tree): the searched disparities iMin .. iMin + iRange - 1. */
struct _SDisparityConfig {
    int iMin = 0;
    int iRange = 0;
    void Set(int _iMin, int _iRange) {
        iMin = _iMin;
        iRange = _iRange;
    }
};

/* ---- device images --------------------------------------------------------- */

/* A non-owning view of a pitched device image (trivially copyable, like the
 * reference's _CDeviceSurface). An empty view (ptr null) stands for the
 * reference's unused xImageDispInit / xImageDebug arguments. */
class _CDeviceSurface {
public:
    _CDeviceSurface() = default;
    _CDeviceSurface(void* ptr, size_t pitch_bytes, const SImageFormat& f) : m_xFormat(f) {
        m_xImage = ct_image{ptr, pitch_bytes, f.iWidth, f.iHeight, static_cast<int32_t>(f.eDataType), 0};
    }

    bool IsValid() const { return m_xImage.ptr != nullptr; }
    const SImageFormat& Format() const { return m_xFormat; }
    void* DataPointer() const { return m_xImage.ptr; }
    size_t Pitch() const { return m_xImage.pitch_bytes; }
    const ct_image* C() const { return IsValid() ? &m_xImage : nullptr; }

protected:
    ct_image m_xImage{nullptr, 0, 0, 0, 0, 0};
    SImageFormat m_xFormat;
};

/* An owning pitched device image (cudaMallocPitch), the role of the
 * reference's CDeviceSurface::Create / CopyFrom / CopyInto. Caller memory:
 * the library never allocates the images it is given. */
class CDeviceSurface : public _CDeviceSurface {
public:
    CDeviceSurface() = default;
    explicit CDeviceSurface(const SImageFormat& f) { Create(f); }
    ~CDeviceSurface() { Destroy(); }
    CDeviceSurface(const CDeviceSurface&) = delete;
    CDeviceSurface& operator=(const CDeviceSurface&) = delete;
    CDeviceSurface(CDeviceSurface&& o) noexcept { *this = std::move(o); }
    CDeviceSurface& operator=(CDeviceSurface&& o) noexcept {
        if (this != &o) {
            Destroy();
            m_xImage = o.m_xImage;
            m_xFormat = o.m_xFormat;
            o.m_xImage.ptr = nullptr;
        }
        return *this;
    }

    void Create(const SImageFormat& f) {
        Destroy();
        void* p = nullptr;
        size_t pitch = 0;
        EnsureCuda(cudaMallocPitch(&p, &pitch, size_t(f.iWidth) * BytesPerPixel(f.eDataType), size_t(f.iHeight)),
                   "CDeviceSurface::Create");
        m_xFormat = f;
        m_xImage = ct_image{p, pitch, f.iWidth, f.iHeight, static_cast<int32_t>(f.eDataType), 0};
    }

    void Destroy() {
        if (m_xImage.ptr) cudaFree(m_xImage.ptr);
        m_xImage.ptr = nullptr;
    }

    /* Host rows of host_pitch bytes (0: tightly packed). Synchronous. */
    void CopyFrom(const void* host, size_t host_pitch = 0) {
        const size_t row = size_t(m_xFormat.iWidth) * BytesPerPixel(m_xFormat.eDataType);
        EnsureCuda(cudaMemcpy2D(m_xImage.ptr, m_xImage.pitch_bytes, host, host_pitch ? host_pitch : row, row,
                                size_t(m_xFormat.iHeight), cudaMemcpyHostToDevice),
                   "CDeviceSurface::CopyFrom");
    }

    void CopyInto(void* host, size_t host_pitch = 0) const {
        const size_t row = size_t(m_xFormat.iWidth) * BytesPerPixel(m_xFormat.eDataType);
        EnsureCuda(cudaMemcpy2D(host, host_pitch ? host_pitch : row, m_xImage.ptr, m_xImage.pitch_bytes, row,
                                size_t(m_xFormat.iHeight), cudaMemcpyDeviceToHost),
                   "CDeviceSurface::CopyInto");
    }

    template <typename T>
    std::vector<T> CopyInto() const {
        std::vector<T> v(size_t(m_xFormat.iWidth) * size_t(m_xFormat.iHeight));
        if (sizeof(T) != BytesPerPixel(m_xFormat.eDataType)) throw CError(CT_ETYPE, "CopyInto: element size");
        CopyInto(v.data());
        return v;
    }
};

/* ---- driver base and ProcessKernel ----------------------------------------- */

class CKernelDriverBase {
public:
    explicit CKernelDriverBase(const char* name) : m_sKernelName(name) {}
    ~CKernelDriverBase() {
        if (m_evStart) cudaEventDestroy(m_evStart);
        if (m_evStop) cudaEventDestroy(m_evStop);
        ct_destroy(m_pHandle);
    }
    CKernelDriverBase(const CKernelDriverBase&) = delete;
    CKernelDriverBase& operator=(const CKernelDriverBase&) = delete;

    const std::string& KernelName() const { return m_sKernelName; }
    void SetStream(cudaStream_t s) { m_xStream = s; }
    cudaStream_t Stream() const { return m_xStream; }
    ct_handle* Handle() const { return m_pHandle; }
    double LastProcessTime() const { return m_dLastProcessTime; }

    /* Event before / after Process on the driver's stream; End waits and
     * stores the elapsed milliseconds (KernelDriverBase.h:139-148). */
    void Begin() {
        if (!m_evStart) {
            EnsureCuda(cudaEventCreate(&m_evStart), "cudaEventCreate");
            EnsureCuda(cudaEventCreate(&m_evStop), "cudaEventCreate");
        }
        EnsureCuda(cudaEventRecord(m_evStart, m_xStream), "Begin");
    }
    void End() {
        EnsureCuda(cudaEventRecord(m_evStop, m_xStream), "End");
        EnsureCuda(cudaEventSynchronize(m_evStop), "End");
        float ms = 0.f;
        EnsureCuda(cudaEventElapsedTime(&ms, m_evStart, m_evStop), "End");
        m_dLastProcessTime = ms;
    }
    /* Reads (and clears) the device status word of the handle's launches; a
     * bounded device-side wait that gave up becomes CError(CT_ETIMEOUT). */
    void EnsureDeviceStatus() {
        if (!m_pHandle) return;  // drivers whose only path has no device-side waits
        int32_t st = 0;
        Ensure(ct_handle_device_status(m_pHandle, &st), m_sKernelName.c_str());
        if (st != 0) throw CError(st, m_sKernelName + ": device status " + std::to_string(st));
    }

protected:
    ct_handle* EnsureHandle(int (*create)(ct_handle**)) {
        if (!m_pHandle) Ensure(create(&m_pHandle), m_sKernelName.c_str());
        return m_pHandle;
    }
    ct_stream S() const { return reinterpret_cast<ct_stream>(m_xStream); }

    ct_handle* m_pHandle = nullptr;
    cudaStream_t m_xStream = nullptr;
    cudaEvent_t m_evStart = nullptr;
    cudaEvent_t m_evStop = nullptr;
    double m_dLastProcessTime = 0.0;
    std::string m_sKernelName;
};

/* Runs xDriver.Process(args...) between Begin and End and returns the
 * milliseconds it took on the device (KernelDriverBase.h:180-199). */
template <typename TDriver, typename... TPars>
double ProcessKernel(TDriver& xDriver, TPars&&... xPars) {
    xDriver.Begin();
    xDriver.Process(std::forward<TPars>(xPars)...);
    xDriver.End();
    xDriver.EnsureDeviceStatus();
    return xDriver.LastProcessTime();
}

namespace detail {
inline void RequireInputFormat(const SImageFormat& f, const char* who) {
    if (f.eDataType != EDataType::UInt8)
        throw CError(CT_ETYPE, std::string(who) + ": input images must be UInt8 luminance");
}
inline void RequireDispConfig(const _SDisparityConfig& c, const char* who) {
    if (c.iMin < 0) throw CError(CT_EINVAL, std::string(who) + ": iMin must be >= 0");
}
/* The ID thresholds act on the reference's 4 x uint16 output only. */
inline void RejectIdThresholds(bool bAnySet, const char* who) {
    if (bAnySet)
        throw CError(CT_EINVAL, std::string(who) +
                                    ": the ID thresholds label the 4 x uint16 output, not the plain disparity map");
}

/* A reference-compat matcher handle (ct_bm_compat_*) owned by a driver:
 * the path that writes the reference's 4 x uint16 TPixelEx output. */
class CCompat {
public:
    CCompat() = default;
    ~CCompat() { ct_destroy(m_pHandle); }
    CCompat(const CCompat&) = delete;
    CCompat& operator=(const CCompat&) = delete;
    void Configure(int iDevice, const ct_format& f, const ct_compat_params& p, const char* who) {
        if (!m_pHandle) Ensure(ct_bm_compat_create(&m_pHandle), who);
        Ensure(ct_bm_compat_configure(m_pHandle, iDevice, &f, &p), who);
        m_bConfigured = true;
    }
    bool IsConfigured() const { return m_bConfigured; }
    void Process(const ct_image* disp, const ct_image* l, const ct_image* r, ct_stream s, const char* who) {
        if (!m_bConfigured) throw CError(CT_ESTATE, std::string(who) + ": this configuration has no 4 x uint16 output");
        Ensure(ct_bm_compat_process(m_pHandle, disp, l, r, s), who);
    }
    ct_handle* Handle() const { return m_pHandle; }

private:
    ct_handle* m_pHandle = nullptr;
    bool m_bConfigured = false;
};

inline ct_compat_params CompatParams(int32_t method, int32_t range, int32_t dmin, int32_t patch, int32_t sim,
                                     bool bLeftToRight, float fGrad, float fScore, float fDelta) {
    ct_compat_params p{};
    p.method = method;
    p.disp_count = range;
    p.disp_min = dmin;
    p.patch = patch;
    p.sim_type = sim;
    p.left_to_right = bLeftToRight ? 1 : 0;
    p.grad_thresh = fGrad;
    p.score_thresh = fScore;
    p.min_delta_thresh = fDelta;
    return p;
}

inline bool IsU16x4(const _CDeviceSurface& x) { return x.Format().eDataType == EDataType::UInt16x4; }
}  // namespace detail

/* ---- CensusTransform (CensusTransform.h:44-70) ----------------------------- */
namespace CensusTransform {

enum class EWindow : int32_t { Census_9x7 = CT_CENSUS_9X7, Census_3x3 = CT_CENSUS_3X3 };

class CDriver : public CKernelDriverBase {
public:
    CDriver() : CKernelDriverBase("Census Transform") {}

    /* Census_9x7 (U8 -> U64, the matcher's descriptor) by default;
     * Census_3x3 is the reference's transform exactly (U8 -> U8). */
    void Configure(const CDevice& xDevice, const SImageFormat& xFormat, EWindow eWindow = EWindow::Census_9x7) {
        detail::RequireInputFormat(xFormat, "CensusTransform");
        EnsureHandle(ct_census_create);
        const ct_format f = xFormat.ToC();
        const ct_census_params p{static_cast<int32_t>(eWindow)};
        Ensure(ct_census_configure(m_pHandle, xDevice.iDevice, &f, &p), "CensusTransform::Configure");
    }

    void Process(_CDeviceSurface& xImageTrg, const _CDeviceSurface& xImageSrc) {
        Ensure(ct_census_process(m_pHandle, xImageTrg.C(), xImageSrc.C(), S()), "CensusTransform::Process");
    }
};

}  // namespace CensusTransform

/* ---- BlockMatcherSAD1 (BlockMatcherSAD1.h:42-127) -------------------------- */
namespace BlockMatcherSAD1 {

/* Patch_16x16 (the reference's configuration) feeds the 4 x uint16 output;
 * the plain exhaustive matcher takes the odd windows 3x3 .. 9x9. */
enum class EConfig { Patch_16x16 = 0, Patch_3x3, Patch_5x5, Patch_7x7, Patch_9x9 };

struct SParameter {
    int iOffset = 0;
    int iDispRange = 0;
    float fSadThresh = 0.f;
    int iMinDeltaThresh = 0;
    float fGradThresh = 0.f;
    EConfig eConfig = EConfig::Patch_9x9;
    bool bLeftToRight = true;

    void Set(int _iOffset, int _iDispRange, int _iMinDeltaThresh, float _fSadThresh, float _fGradThresh,
             EConfig _eConfig) {
        iOffset = _iOffset;
        iDispRange = _iDispRange;
        iMinDeltaThresh = _iMinDeltaThresh;
        fSadThresh = _fSadThresh;
        fGradThresh = _fGradThresh;
        eConfig = _eConfig;
    }
};

/* Process into a UInt16x4 surface: the reference's coarse / fine search with
 * its gates and IDs (ct_bm_compat_*, CT_COMPAT_SAD1). Into UInt8 / UInt16:
 * the exhaustive winner-take-all over all disparities with the gradient gate;
 * the ID thresholds (fSadThresh, iMinDeltaThresh) must then be 0. */
class CDriver : public CKernelDriverBase {
public:
    CDriver() : CKernelDriverBase("Block Matcher SAD 1") {}

    void Configure(const CDevice& xDevice, const SImageFormat& xFormat, const SParameter& xPars) {
        detail::RequireInputFormat(xFormat, "BlockMatcherSAD1");
        if (xPars.iOffset < 0) throw CError(CT_EINVAL, "BlockMatcherSAD1: iOffset must be >= 0");
        m_xPars = xPars;
        const ct_format f = xFormat.ToC();
        const int patch = xPars.eConfig == EConfig::Patch_16x16 ? 16 : 2 * static_cast<int>(xPars.eConfig) + 1;
        m_xCompat.Configure(xDevice.iDevice, f,
                            detail::CompatParams(CT_COMPAT_SAD1, xPars.iDispRange, xPars.iOffset, patch, 0,
                                                 xPars.bLeftToRight, xPars.fGradThresh, xPars.fSadThresh,
                                                 float(xPars.iMinDeltaThresh)),
                            "BlockMatcherSAD1::Configure");
        if (xPars.eConfig != EConfig::Patch_16x16) {
            EnsureHandle(ct_bm_sad_create);
            const ct_sad_params p{xPars.iDispRange, static_cast<int32_t>(xPars.eConfig), xPars.bLeftToRight ? 1 : 0,
                                  xPars.iOffset};
            Ensure(ct_bm_sad_configure(m_pHandle, xDevice.iDevice, &f, &p), "BlockMatcherSAD1::Configure");
            Ensure(ct_bm_set_gradient_gate(m_pHandle, xPars.fGradThresh), "BlockMatcherSAD1::Configure");
        }
    }

    /* xImageDisp: UInt16x4 (reference output) or UInt8 / UInt16 (plain map). */
    void Process(_CDeviceSurface& xImageDisp, const _CDeviceSurface& xImageL, const _CDeviceSurface& xImageR) {
        if (detail::IsU16x4(xImageDisp)) {
            m_xCompat.Process(xImageDisp.C(), xImageL.C(), xImageR.C(), S(), "BlockMatcherSAD1::Process");
            return;
        }
        if (m_xPars.eConfig == EConfig::Patch_16x16)
            throw CError(CT_EINVAL, "BlockMatcherSAD1: Patch_16x16 writes the UInt16x4 output only");
        detail::RejectIdThresholds(m_xPars.fSadThresh != 0.f || m_xPars.iMinDeltaThresh != 0, "BlockMatcherSAD1");
        Ensure(ct_bm_sad_process(m_pHandle, xImageDisp.C(), xImageL.C(), xImageR.C(), S()),
               "BlockMatcherSAD1::Process");
    }

private:
    SParameter m_xPars;
    detail::CCompat m_xCompat;
};

}  // namespace BlockMatcherSAD1

/* ---- BlockMatcherNCC (BlockMatcherNCC.h:41-144) ---------------------------- */
namespace BlockMatcherNCC {

enum class EConfig { Patch_11x11 = 0, Patch_9x9, Patch_5x5 };

struct SParameter {
    _SDisparityConfig xDispConfig;
    int iMinDeltaThresh = 0;
    float fNccThresh = 0.f;
    float fGradThresh = 0.f;
    int iUseDispInput = 0;
    EConfig eConfig = EConfig::Patch_11x11;
    bool bLeftToRight = true;

    void Set(const _SDisparityConfig& _xDispConfig, int _iMinDeltaThresh, float _fNccThresh, float _fGradThresh,
             int _iUseDispInput, bool _bLeftToRight, EConfig _eConfig) {
        xDispConfig = _xDispConfig;
        iMinDeltaThresh = _iMinDeltaThresh;
        fNccThresh = _fNccThresh;
        fGradThresh = _fGradThresh;
        iUseDispInput = _iUseDispInput;
        bLeftToRight = _bLeftToRight;
        eConfig = _eConfig;
    }
};

/* Process into UInt16x4: the reference's uint8-quantised NCC with its
 * gates, IDs and specificity channels (CT_COMPAT_NCC, either direction).
 * Into UInt8 / UInt16 (+ Single score in xImageDebug): the FP32 NCC
 * winner-take-all (left-to-right), optionally guided, with the gradient gate;
 * fNccThresh and iMinDeltaThresh must then be 0. */
class CDriver : public CKernelDriverBase {
public:
    CDriver() : CKernelDriverBase("Block Matcher NCC") {}

    void Configure(const CDevice& xDevice, const SImageFormat& xFormat, const SParameter& xPars) {
        detail::RequireInputFormat(xFormat, "BlockMatcherNCC");
        detail::RequireDispConfig(xPars.xDispConfig, "BlockMatcherNCC");
        m_xPars = xPars;
        m_bUseDispInput = xPars.iUseDispInput != 0;
        static const int32_t radius[] = {5, 4, 2};
        const int r = radius[static_cast<int>(xPars.eConfig)];
        const ct_format f = xFormat.ToC();
        m_xCompat.Configure(xDevice.iDevice, f,
                            detail::CompatParams(CT_COMPAT_NCC, xPars.xDispConfig.iRange, xPars.xDispConfig.iMin,
                                                 2 * r + 1, 0, xPars.bLeftToRight, xPars.fGradThresh,
                                                 xPars.fNccThresh, float(xPars.iMinDeltaThresh)),
                            "BlockMatcherNCC::Configure");
        if (xPars.bLeftToRight) {  // the plain FP32 matcher is left-to-right
            EnsureHandle(ct_bm_ncc_create);
            const ct_ncc_params p{xPars.xDispConfig.iRange, r, 1, xPars.xDispConfig.iMin};
            Ensure(ct_bm_ncc_configure(m_pHandle, xDevice.iDevice, &f, &p), "BlockMatcherNCC::Configure");
            Ensure(ct_bm_set_gradient_gate(m_pHandle, xPars.fGradThresh), "BlockMatcherNCC::Configure");
        }
    }

    /* xImageDisp: UInt16x4 (reference output) or UInt8 / UInt16; xImageDebug,
     * when valid, receives the Single NCC score of the plain matcher. With
     * iUseDispInput set, xImageDispInit is the coarse disparity map of the
     * guided mode (MatcherUseDisparity; see ct_bm_ncc_process); without it,
     * xImageDispInit is ignored. */
    void Process(_CDeviceSurface& xImageDisp, const _CDeviceSurface& xImageL, const _CDeviceSurface& xImageR,
                 const _CDeviceSurface& xImageDispInit, const _CDeviceSurface& xImageDebug) {
        if (detail::IsU16x4(xImageDisp)) {
            if (m_bUseDispInput)
                throw CError(CT_EINVAL, "BlockMatcherNCC: the guided mode writes the plain maps only");
            m_xCompat.Process(xImageDisp.C(), xImageL.C(), xImageR.C(), S(), "BlockMatcherNCC::Process");
            return;
        }
        if (!m_pHandle) throw CError(CT_EINVAL, "BlockMatcherNCC: right-to-left writes the UInt16x4 output only");
        detail::RejectIdThresholds(m_xPars.fNccThresh != 0.f || m_xPars.iMinDeltaThresh != 0, "BlockMatcherNCC");
        if (m_bUseDispInput && !xImageDispInit.IsValid())
            throw CError(CT_EINVAL, "BlockMatcherNCC: iUseDispInput needs xImageDispInit");
        Ensure(ct_bm_ncc_process(m_pHandle, xImageDisp.C(), xImageDebug.C(), xImageL.C(), xImageR.C(),
                                 m_bUseDispInput ? xImageDispInit.C() : nullptr, S()),
               "BlockMatcherNCC::Process");
    }
    void Process(_CDeviceSurface& xImageDisp, const _CDeviceSurface& xImageL, const _CDeviceSurface& xImageR) {
        Process(xImageDisp, xImageL, xImageR, _CDeviceSurface(), _CDeviceSurface());
    }
    /* Unguided plain matching with the window sums on the tensor cores (the
     * default) or on the CUDA cores; the maps and scores are the same. */
    void SetTensorCores(bool bEnable) {
        if (!m_pHandle) throw CError(CT_ESTATE, "BlockMatcherNCC: configure a left-to-right matcher first");
        Ensure(ct_bm_ncc_set_tensor_cores(m_pHandle, bEnable ? 1 : 0), "BlockMatcherNCC::SetTensorCores");
    }

private:
    SParameter m_xPars;
    bool m_bUseDispInput = false;
    detail::CCompat m_xCompat;
};

}  // namespace BlockMatcherNCC

/* ---- BlockMatcherAW1 (BlockMatcherAW1.h:41-157) ---------------------------- */
namespace BlockMatcherAW1 {

/* Patch_15x15 / Patch_9x9: the reference's centre + best 2 of 4 sub-window
 * score (5 x 5 / 3 x 3 sub-windows) with its gates and IDs, written as the
 * UInt16x4 output or its x channel into UInt16 (CT_COMPAT_AW1).
 * Shifted5_7x7: minimum of the 7x7 SAD over the centred window and the
 * windows shifted by +-3 px in x and y, with FP32 sub-pixel refinement. */
enum class EConfig { Patch_15x15 = 0, Patch_9x9, Shifted5_7x7 };
enum class ESimType { AbsoluteDifference = 0, SignedProduct };

struct SParameter {
    _SDisparityConfig xDispConfig;
    float fMinDeltaThresh = 0.f;
    float fSimThresh = 0.f;
    float fGradThresh = 0.f;
    int iUseDispInput = 0;
    EConfig eConfig = EConfig::Shifted5_7x7;
    ESimType eSimType = ESimType::AbsoluteDifference;
    bool bLeftToRight = true;

    void Set(const _SDisparityConfig& _xDispConfig, float _fMinDeltaThresh, float _fSimThresh, float _fGradThresh,
             int _iUseDispInput, bool _bLeftToRight, EConfig _eConfig, ESimType _eSimType) {
        xDispConfig = _xDispConfig;
        fMinDeltaThresh = _fMinDeltaThresh;
        fSimThresh = _fSimThresh;
        fGradThresh = _fGradThresh;
        iUseDispInput = _iUseDispInput;
        bLeftToRight = _bLeftToRight;
        eConfig = _eConfig;
        eSimType = _eSimType;
    }
};

class CDriver : public CKernelDriverBase {
public:
    CDriver() : CKernelDriverBase("Block Matcher Adaptive Window 1") {}

    void Configure(const CDevice& xDevice, const SImageFormat& xFormat, const SParameter& xPars) {
        detail::RequireInputFormat(xFormat, "BlockMatcherAW1");
        detail::RequireDispConfig(xPars.xDispConfig, "BlockMatcherAW1");
        m_xPars = xPars;
        m_bUseDispInput = xPars.iUseDispInput != 0;
        const ct_format f = xFormat.ToC();
        if (xPars.eConfig != EConfig::Shifted5_7x7) {
            if (m_bUseDispInput) throw CError(CT_EINVAL, "BlockMatcherAW1: the guided mode is built for Shifted5_7x7");
            m_xCompat.Configure(
                xDevice.iDevice, f,
                detail::CompatParams(CT_COMPAT_AW1, xPars.xDispConfig.iRange, xPars.xDispConfig.iMin,
                                     xPars.eConfig == EConfig::Patch_15x15 ? 5 : 3,
                                     xPars.eSimType == ESimType::SignedProduct ? 1 : 0, xPars.bLeftToRight,
                                     xPars.fGradThresh, xPars.fSimThresh, xPars.fMinDeltaThresh),
                "BlockMatcherAW1::Configure");
            return;
        }
        if (xPars.eSimType != ESimType::AbsoluteDifference)
            throw CError(CT_EINVAL, "BlockMatcherAW1: Shifted5_7x7 is an absolute-difference cost");
        detail::RejectIdThresholds(xPars.fSimThresh != 0.f || xPars.fMinDeltaThresh != 0.f, "BlockMatcherAW1");
        EnsureHandle(ct_bm_aw_create);
        const ct_aw_params p{xPars.xDispConfig.iRange, xPars.bLeftToRight ? 1 : 0, xPars.xDispConfig.iMin, 0};
        Ensure(ct_bm_aw_configure(m_pHandle, xDevice.iDevice, &f, &p), "BlockMatcherAW1::Configure");
        Ensure(ct_bm_set_gradient_gate(m_pHandle, xPars.fGradThresh), "BlockMatcherAW1::Configure");
    }

    /* Patch_15x15 / Patch_9x9: xImageDisp UInt16x4 (reference output) or
     * UInt16 (its x channel). Shifted5_7x7: Single (sub-pixel, -1 invalid) or
     * UInt8 / UInt16 (integer winner-take-all); with iUseDispInput set,
     * xImageDispInit is the coarse map of the guided mode
     * (ct_bm_aw_process_guided). xImageDebug is unused. */
    void Process(_CDeviceSurface& xImageDisp, const _CDeviceSurface& xImageL, const _CDeviceSurface& xImageR,
                 const _CDeviceSurface& xImageDispInit, const _CDeviceSurface& /*xImageDebug*/) {
        if (m_xPars.eConfig != EConfig::Shifted5_7x7) {
            m_xCompat.Process(xImageDisp.C(), xImageL.C(), xImageR.C(), S(), "BlockMatcherAW1::Process");
            return;
        }
        if (!m_bUseDispInput) {
            Ensure(ct_bm_aw_process(m_pHandle, xImageDisp.C(), xImageL.C(), xImageR.C(), S()),
                   "BlockMatcherAW1::Process");
            return;
        }
        if (!xImageDispInit.IsValid()) throw CError(CT_EINVAL, "BlockMatcherAW1: iUseDispInput needs xImageDispInit");
        Ensure(ct_bm_aw_process_guided(m_pHandle, xImageDisp.C(), xImageL.C(), xImageR.C(), xImageDispInit.C(), S()),
               "BlockMatcherAW1::Process");
    }
    void Process(_CDeviceSurface& xImageDisp, const _CDeviceSurface& xImageL, const _CDeviceSurface& xImageR) {
        Process(xImageDisp, xImageL, xImageR, _CDeviceSurface(), _CDeviceSurface());
    }

private:
    SParameter m_xPars;
    bool m_bUseDispInput = false;
    detail::CCompat m_xCompat;
};

}  // namespace BlockMatcherAW1

/* ---- BlockMatcherAW2 (BlockMatcherAW2.h:41-135) ---------------------------- */
namespace BlockMatcherAW2 {

/* Centre + 2 lowest of 4 sub-window SADs (5 x 5 / 3 x 3 sub-windows),
 * scanned from the largest disparity (CT_COMPAT_AW2). The reference centres
 * its range on iOffset (x_R = x - iOffset - iDispRange / 2 + idx,
 * BlockMatcherAW2.cu:539); here iOffset is the smallest disparity and the
 * range never goes below 0. */
enum class EConfig { Patch_15x15 = 0, Patch_9x9 };

struct SParameter {
    int iOffset = 0;
    int iDispRange = 0;
    int iMinDeltaThresh = 0;
    float fSadThresh = 0.f;
    float fGradThresh = 0.f;
    int iUseDispInput = 0;
    EConfig eConfig = EConfig::Patch_9x9;

    void Set(int _iOffset, int _iDispRange, int _iMinDeltaThresh, float _fSadThresh, float _fGradThresh,
             int _iUseDispInput, EConfig _eConfig) {
        iOffset = _iOffset;
        iDispRange = _iDispRange;
        iMinDeltaThresh = _iMinDeltaThresh;
        fSadThresh = _fSadThresh;
        fGradThresh = _fGradThresh;
        iUseDispInput = _iUseDispInput;
        eConfig = _eConfig;
    }
};

class CDriver : public CKernelDriverBase {
public:
    CDriver() : CKernelDriverBase("Block Matcher Adaptive Window 2") {}

    void Configure(const CDevice& xDevice, const SImageFormat& xFormat, const SParameter& xPars) {
        detail::RequireInputFormat(xFormat, "BlockMatcherAW2");
        if (xPars.iOffset < 0) throw CError(CT_EINVAL, "BlockMatcherAW2: iOffset must be >= 0");
        if (xPars.iUseDispInput) throw CError(CT_EINVAL, "BlockMatcherAW2: the guided mode is not built");
        m_xCompat.Configure(xDevice.iDevice, xFormat.ToC(),
                            detail::CompatParams(CT_COMPAT_AW2, xPars.iDispRange, xPars.iOffset,
                                                 xPars.eConfig == EConfig::Patch_15x15 ? 5 : 3, 0, true,
                                                 xPars.fGradThresh, xPars.fSadThresh, float(xPars.iMinDeltaThresh)),
                            "BlockMatcherAW2::Configure");
    }

    /* xImageDisp: UInt16x4 (reference output) or UInt16 (its x channel). */
    void Process(_CDeviceSurface& xImageDisp, const _CDeviceSurface& xImageL, const _CDeviceSurface& xImageR,
                 const _CDeviceSurface& /*xImageDispInit*/ = _CDeviceSurface()) {
        m_xCompat.Process(xImageDisp.C(), xImageL.C(), xImageR.C(), S(), "BlockMatcherAW2::Process");
    }

private:
    detail::CCompat m_xCompat;
};

}  // namespace BlockMatcherAW2

/* ---- BlockMatcher1 (BlockMatcher1.h:41-190) -------------------------------- */
namespace BlockMatcher1 {

/* Plain P x P window of (255 - |a - b|) >> 1 (AbsoluteDifference) or the
 * signed product x 127 (SignedProduct), argmax with the reference's scan
 * bookkeeping, gates and IDs (CT_COMPAT_BM1). */
enum class EConfig { Patch_5x5 = 0, Patch_9x9, Patch_11x11, Patch_15x15 };
enum class ESimType { AbsoluteDifference = 0, SignedProduct };

struct SParameter {
    _SDisparityConfig xDispConfig;
    float fMinDeltaThresh = 0.f;
    float fSimThresh = 0.f;
    float fGradThresh = 0.f;
    int iUseDispInput = 0;
    EConfig eConfig = EConfig::Patch_9x9;
    ESimType eSimType = ESimType::AbsoluteDifference;
    bool bLeftToRight = true;

    void Set(const _SDisparityConfig& _xDispConfig, float _fMinDeltaThresh, float _fSimThresh, float _fGradThresh,
             int _iUseDispInput, bool _bLeftToRight, EConfig _eConfig, ESimType _eSimType) {
        xDispConfig = _xDispConfig;
        fMinDeltaThresh = _fMinDeltaThresh;
        fSimThresh = _fSimThresh;
        fGradThresh = _fGradThresh;
        iUseDispInput = _iUseDispInput;
        bLeftToRight = _bLeftToRight;
        eConfig = _eConfig;
        eSimType = _eSimType;
    }
};

class CDriver : public CKernelDriverBase {
public:
    CDriver() : CKernelDriverBase("Block Matcher 1") {}

    void Configure(const CDevice& xDevice, const SImageFormat& xFormat, const SParameter& xPars) {
        detail::RequireInputFormat(xFormat, "BlockMatcher1");
        detail::RequireDispConfig(xPars.xDispConfig, "BlockMatcher1");
        if (xPars.iUseDispInput) throw CError(CT_EINVAL, "BlockMatcher1: the guided mode is not built");
        static const int32_t patch[] = {5, 9, 11, 15};
        m_xCompat.Configure(xDevice.iDevice, xFormat.ToC(),
                            detail::CompatParams(CT_COMPAT_BM1, xPars.xDispConfig.iRange, xPars.xDispConfig.iMin,
                                                 patch[static_cast<int>(xPars.eConfig)],
                                                 xPars.eSimType == ESimType::SignedProduct ? 1 : 0, xPars.bLeftToRight,
                                                 xPars.fGradThresh, xPars.fSimThresh, xPars.fMinDeltaThresh),
                            "BlockMatcher1::Configure");
    }

    /* xImageDisp: UInt16x4 (reference output) or UInt16 (its x channel). */
    void Process(_CDeviceSurface& xImageDisp, const _CDeviceSurface& xImageL, const _CDeviceSurface& xImageR,
                 const _CDeviceSurface& /*xImageDispInit*/ = _CDeviceSurface(),
                 const _CDeviceSurface& /*xImageDebug*/ = _CDeviceSurface()) {
        m_xCompat.Process(xImageDisp.C(), xImageL.C(), xImageR.C(), S(), "BlockMatcher1::Process");
    }

private:
    detail::CCompat m_xCompat;
};

}  // namespace BlockMatcher1

/* ---- CrossCheckDisparityMaps (CrossCheckDisparityMaps.h:38-117) ------------- */
namespace CrossCheckDisparityMaps {

struct SParameter {
    _SDisparityConfig xDispConfig;
    int iDispDeltaThresh = 1;
    int iIsLeftToRight = 1;

    void Set(const _SDisparityConfig& _xDispConfig, int _iDispDeltaThresh, int _iIsLeftToRight) {
        xDispConfig = _xDispConfig;
        iDispDeltaThresh = _iDispDeltaThresh;
        iIsLeftToRight = _iIsLeftToRight;
    }
};

class CDriver : public CKernelDriverBase {
public:
    CDriver() : CKernelDriverBase("Cross Check Disparity Maps") {}

    /* xFormat: the disparity maps' format (UInt8 or UInt16). */
    void Configure(const CDevice& xDevice, const SImageFormat& xFormat, const SParameter& xPars) {
        detail::RequireDispConfig(xPars.xDispConfig, "CrossCheckDisparityMaps");
        EnsureHandle(ct_crosscheck_create);
        const ct_format f = xFormat.ToC();
        const ct_crosscheck_params p{xPars.iDispDeltaThresh, xPars.iIsLeftToRight, 0, 0};
        Ensure(ct_crosscheck_configure(m_pHandle, xDevice.iDevice, &f, &p), "CrossCheckDisparityMaps::Configure");
    }

    void Process(_CDeviceSurface& xDispResult, const _CDeviceSurface& xDispLR, const _CDeviceSurface& xDispRL) {
        Ensure(ct_crosscheck_process(m_pHandle, xDispResult.C(), xDispLR.C(), xDispRL.C(), S()),
               "CrossCheckDisparityMaps::Process");
        m_bRangeRead = false;
    }

    /* Smallest / largest kept disparity of the last Process (min > max when
     * none was kept). The first call after Process synchronises its stream. */
    int DispMin() { return Range().first; }
    int DispMax() { return Range().second; }

private:
    std::pair<int, int> Range() {
        if (!m_bRangeRead) {
            int32_t lo = 0, hi = 0;
            Ensure(ct_crosscheck_range(m_pHandle, &lo, &hi), "CrossCheckDisparityMaps::DispMin/DispMax");
            m_xRange = {lo, hi};
            m_bRangeRead = true;
        }
        return m_xRange;
    }
    bool m_bRangeRead = false;
    std::pair<int, int> m_xRange{0, -1};
};

}  // namespace CrossCheckDisparityMaps

/* ---- ColorDisparityImage (ColorDisparityImage.h:37-120) -------------------- */
namespace ColorDisparityImage {

enum class EStyle : int32_t {
    Analysis = CT_COLOR_ANALYSIS,
    Gray = CT_COLOR_GRAY,
    Color = CT_COLOR_COLOR,
    DispAbs = CT_COLOR_DISP_ABS,
    DispRel = CT_COLOR_DISP_REL,
};

/* Colours are RGBA8 words, r in the low byte (pixUnknown ..
 * pixInconsistent); the defaults are the reference's. */
struct SParameter {
    uint16_t uDispMin = CT_DISP_FIRST, uDispMax = CT_DISP_LAST, uDispInfOffset = 0;
    uint32_t pixUnknown, pixCannotEvaluate, pixSaturated, pixNotSpecific, pixNotFound, pixNotUnique, pixInconsistent;

    SParameter() {
        ct_color_params d;
        Ensure(ct_color_params_default(CT_COLOR_ANALYSIS, &d), "ColorDisparityImage::SParameter");
        pixUnknown = d.colors[0];
        pixCannotEvaluate = d.colors[1];
        pixSaturated = d.colors[2];
        pixNotSpecific = d.colors[3];
        pixNotFound = d.colors[4];
        pixNotUnique = d.colors[5];
        pixInconsistent = d.colors[6];
    }
    void Set(uint16_t _uDispMin, uint16_t _uDispMax, uint16_t _uDispInfOffset) {
        uDispMin = _uDispMin;
        uDispMax = _uDispMax;
        uDispInfOffset = _uDispInfOffset;
    }
};

class CDriver : public CKernelDriverBase {
public:
    CDriver() : CKernelDriverBase("Color Disparity Image") {}

    void Configure(const CDevice& xDevice, const SImageFormat& /*xFormat*/, const SParameter& xPars) {
        m_xPars = xPars;
        EnsureCuda(cudaSetDevice(xDevice.iDevice), "ColorDisparityImage::Configure");
    }

    /* xColorImage: EDataType::RGBA8 for Analysis / Color, UInt16 for the
     * other styles; xDisparityImage: UInt16 codes or UInt8 disparities. */
    void Process(_CDeviceSurface& xColorImage, const _CDeviceSurface& xDisparityImage, EStyle eStyle) {
        ct_color_params p{};
        p.style = static_cast<int32_t>(eStyle);
        p.disp_min = m_xPars.uDispMin;
        p.disp_max = m_xPars.uDispMax;
        p.inf_offset = m_xPars.uDispInfOffset;
        const uint32_t c[7] = {m_xPars.pixUnknown, m_xPars.pixCannotEvaluate, m_xPars.pixSaturated,
                               m_xPars.pixNotSpecific, m_xPars.pixNotFound, m_xPars.pixNotUnique,
                               m_xPars.pixInconsistent};
        for (int i = 0; i < 7; ++i) p.colors[i] = c[i];
        ct_image out = *xColorImage.C();
        if (eStyle == EStyle::Analysis || eStyle == EStyle::Color) out.type = CT_PIX_RGBA8;
        Ensure(ct_color_disparity(&out, xDisparityImage.C(), &p, S()), "ColorDisparityImage::Process");
    }

    void EnsureDeviceStatus() {}  // no device-side waits

private:
    SParameter m_xPars;
};

}  // namespace ColorDisparityImage

/* ---- MapDisparityTo3D (MapDisparityTo3D.h:41-150) ------------------------- */
namespace MapDisparityTo3D {

/* Replaces Clu::Camera::_CStereoPinhole (CluTec.Core, not in the reference
 * tree): the left and right pinhole cameras (ct_pinhole). */
struct CStereoPinhole {
    ct_pinhole cam[2];
};

struct SParameter {
    uint16_t uDispMin = CT_DISP_FIRST, uDispMax = CT_DISP_LAST;
    bool bIsCsRUT = false;  // x right, y up, z towards (else y down, z away)
    CStereoPinhole camStereoPinhole{};
    void Set(uint16_t _uDispMin, uint16_t _uDispMax, bool _bIsCsRUT, const CStereoPinhole& _cam) {
        uDispMin = _uDispMin;
        uDispMax = _uDispMax;
        bIsCsRUT = _bIsCsRUT;
        camStereoPinhole = _cam;
    }
};

class CDriver : public CKernelDriverBase {
public:
    CDriver() : CKernelDriverBase("Map Disparity To 3D") {}

    /* xFormat: the disparity map (UInt16 codes, UInt8 or Single sub-pixel). */
    void Configure(const CDevice& xDevice, const SImageFormat& xFormat, const SParameter& xPars) {
        ct_map3d_params p{};
        p.disp_min = xPars.uDispMin;
        p.disp_max = xPars.uDispMax;
        p.cs_rut = xPars.bIsCsRUT ? 1 : 0;
        p.cam[0] = xPars.camStereoPinhole.cam[0];
        p.cam[1] = xPars.camStereoPinhole.cam[1];
        const ct_format f = xFormat.ToC();
        Ensure(ct_map3d_configure(EnsureHandle(ct_map3d_create), xDevice.iDevice, &f, &p),
               "MapDisparityTo3D::Configure");
    }

    /* surfMap3D: EDataType::RGBA_Single (x, y, z, valid). */
    void Process(_CDeviceSurface& surfMap3D, const _CDeviceSurface& surfDisparity) {
        Ensure(ct_map3d_process(m_pHandle, surfMap3D.C(), surfDisparity.C(), S()), "MapDisparityTo3D::Process");
    }

    /* pixMin / pixMax of the last Process (synchronises). */
    void GetRange(float (&afMin)[3], float (&afMax)[3]) {
        Ensure(ct_map3d_range(m_pHandle, afMin, afMax), "MapDisparityTo3D::GetRange");
    }
};

}  // namespace MapDisparityTo3D

/* ---- CDeviceSurfMipMap (DeviceSurfMipMap.h:40-150) ------------------------- */

/* The packed disparity mip-map: one F32 image holding every level (layout:
 * ct_disp_mipmap_format / ct_disp_mipmap_level). GetMipMap returns a view of
 * one level that any driver taking an F32 image accepts. */
class CDeviceSurfMipMap {
public:
    CDeviceSurfMipMap() = default;
    explicit CDeviceSurfMipMap(const SImageFormat& xFormat) { Create(xFormat); }

    /* xFormat: the format of level 0 (the disparity map's size). */
    void Create(const SImageFormat& xFormat) {
        int32_t pw = 0, n = 0;
        Ensure(ct_disp_mipmap_format(xFormat.iWidth, xFormat.iHeight, &pw, &n), "CDeviceSurfMipMap::Create");
        m_xImage.Create(SImageFormat(pw, xFormat.iHeight, EDataType::Single));
        m_xFormat = SImageFormat(xFormat.iWidth, xFormat.iHeight, EDataType::Single);
        m_iMax = n;
        m_iActive = 0;
    }

    int MaxMipMapLevelCount() const { return m_iMax; }
    int GetActiveMipMapLevelCount() const { return m_iActive; }
    void SetActiveMipMapLevelCount(int iCount) {
        if (iCount < 0 || iCount > m_iMax) throw CError(CT_EINVAL, "Given mip-map level count out of range");
        m_iActive = iCount;
    }

    void GetOrigin(int& iX, int& iY, int iLevel) const {
        int32_t x, y, w, h;
        Ensure(ct_disp_mipmap_level(m_xFormat.iWidth, m_xFormat.iHeight, iLevel, &x, &y, &w, &h), "GetOrigin");
        iX = x;
        iY = y;
    }
    SImageFormat Format(int iLevel) const {
        int32_t x, y, w, h;
        Ensure(ct_disp_mipmap_level(m_xFormat.iWidth, m_xFormat.iHeight, iLevel, &x, &y, &w, &h), "Format");
        return SImageFormat(w, h, EDataType::Single);
    }
    _CDeviceSurface GetMipMap(int iLevel) const {
        int iX = 0, iY = 0;
        GetOrigin(iX, iY, iLevel);
        char* p = static_cast<char*>(m_xImage.DataPointer()) + size_t(iY) * m_xImage.Pitch() + size_t(iX) * 4;
        return _CDeviceSurface(p, m_xImage.Pitch(), Format(iLevel));
    }
    /* The whole packed image. */
    const CDeviceSurface& Surface() const { return m_xImage; }

private:
    CDeviceSurface m_xImage;
    SImageFormat m_xFormat;
    int m_iMax = 0, m_iActive = 0;
};

/* ---- CreateDispMipMaps (CreateDispMipMaps.h:44-80) ------------------------- */
namespace CreateDispMipMaps {

class CDriver : public CKernelDriverBase {
public:
    CDriver() : CKernelDriverBase("Create Disparity Mip Maps") {}

    void Configure(const CDevice& xDevice, const SImageFormat& xFormat) {
        EnsureCuda(cudaSetDevice(xDevice.iDevice), "CreateDispMipMaps::Configure");
        m_xFormat = xFormat;
    }

    /* CDriver::Run (CreateDispMipMaps.cu:246-330): levels 0 .. iLevelCount - 1
     * of xMipMap from surfDisp (UInt16 codes or UInt8 disparities); <= 0 =
     * all, 1 = nothing, more than MaxMipMapLevelCount() throws. xTemp is
     * not used (the horizontal and vertical passes are one kernel). Timed
     * like the reference's Run (LastProcessTime). */
    void Run(CDeviceSurfMipMap& xMipMap, CDeviceSurface& /*xTemp*/, const _CDeviceSurface& surfDisp,
             int iLevelCount = 0) {
        Begin();
        Ensure(ct_disp_mipmaps(xMipMap.Surface().C(), surfDisp.C(), iLevelCount, S()), "CreateDispMipMaps::Run");
        End();
        if (iLevelCount != 1) xMipMap.SetActiveMipMapLevelCount(iLevelCount <= 0 ? xMipMap.MaxMipMapLevelCount()
                                                                                 : iLevelCount);
    }

    void EnsureDeviceStatus() {}  // no device-side waits

private:
    SImageFormat m_xFormat;
};

}  // namespace CreateDispMipMaps

/* ---- no reference counterpart ----------------------------------------------- */

/* Device cost-curve volume for BlockMatcherCensus::ProcessCurves and
 * ConfidenceNet (layout: ct_curves). */
class CCurveVolume {
public:
    CCurveVolume() = default;
    CCurveVolume(int width, int height, int disp_count) { Create(width, height, disp_count); }
    ~CCurveVolume() {
        if (m_xCurves.ptr) cudaFree(m_xCurves.ptr);
    }
    CCurveVolume(const CCurveVolume&) = delete;
    CCurveVolume& operator=(const CCurveVolume&) = delete;

    void Create(int width, int height, int disp_count) {
        if (m_xCurves.ptr) cudaFree(m_xCurves.ptr);
        m_xCurves.ptr = nullptr;
        size_t pitch = 0;
        Ensure(ct_curves_pitch(width, &pitch), "CCurveVolume::Create");
        const size_t rows = size_t(height) * size_t((disp_count + 3) / 4);
        void* p = nullptr;
        EnsureCuda(cudaMalloc(&p, rows * pitch), "CCurveVolume::Create");
        m_xCurves = ct_curves{p, pitch, width, height, disp_count, 0};
    }
    const ct_curves* C() const { return &m_xCurves; }

private:
    ct_curves m_xCurves{nullptr, 0, 0, 0, 0, 0};
};

/* Census pipeline (9x7 census, 5x5 Hamming aggregation, winner-take-all)
 * in one call per direction; ProcessLR adds the other direction and the
 * cross-check, ProcessCurves the cost-curve export. */
namespace BlockMatcherCensus {

struct SParameter {
    _SDisparityConfig xDispConfig;
    int iAggRadius = 2;
    bool bLeftToRight = true;
};

class CDriver : public CKernelDriverBase {
public:
    CDriver() : CKernelDriverBase("Block Matcher Census") {}

    void Configure(const CDevice& xDevice, const SImageFormat& xFormat, const SParameter& xPars) {
        detail::RequireInputFormat(xFormat, "BlockMatcherCensus");
        detail::RequireDispConfig(xPars.xDispConfig, "BlockMatcherCensus");
        EnsureHandle(ct_bm_census_create);
        const ct_format f = xFormat.ToC();
        const ct_census_match_params p{xPars.xDispConfig.iRange, xPars.iAggRadius, xPars.bLeftToRight ? 1 : 0,
                                       xPars.xDispConfig.iMin};
        Ensure(ct_bm_census_configure(m_pHandle, xDevice.iDevice, &f, &p), "BlockMatcherCensus::Configure");
    }

    void Process(_CDeviceSurface& xImageDisp, const _CDeviceSurface& xImageL, const _CDeviceSurface& xImageR) {
        Ensure(ct_bm_census_process(m_pHandle, xImageDisp.C(), xImageL.C(), xImageR.C(), S()),
               "BlockMatcherCensus::Process");
    }

    /* Any of the three outputs may be an empty surface. */
    void ProcessLR(_CDeviceSurface& xDispLR, _CDeviceSurface& xDispRL, _CDeviceSurface& xDispChecked,
                   int iDispDeltaThresh, const _CDeviceSurface& xImageL, const _CDeviceSurface& xImageR) {
        Ensure(ct_bm_census_process_lr(m_pHandle, xDispLR.C(), xDispRL.C(), xDispChecked.C(), iDispDeltaThresh,
                                       xImageL.C(), xImageR.C(), S()),
               "BlockMatcherCensus::ProcessLR");
    }

    void ProcessCurves(_CDeviceSurface& xImageDisp, CCurveVolume& xCurves, const _CDeviceSurface& xImageL,
                       const _CDeviceSurface& xImageR) {
        Ensure(ct_bm_census_process_curves(m_pHandle, xImageDisp.C(), xCurves.C(), xImageL.C(), xImageR.C(), S()),
               "BlockMatcherCensus::ProcessCurves");
    }

    /* ProcessLR in one matching pass (default) or in two, one per direction;
     * the maps are identical. */
    void SetFusedLR(bool bEnable) {
        Ensure(ct_bm_census_set_fused_lr(m_pHandle, bEnable ? 1 : 0), "BlockMatcherCensus::SetFusedLR");
    }
};

}  // namespace BlockMatcherCensus

/* A stream of frames in host memory: census both ways + cross-check per
 * frame, uploads and downloads of neighbouring frames overlapping the
 * matching. Host buffers must stay valid (inputs unchanged) until Wait for
 * their frame; page-locked memory lets the copies overlap. */
namespace CensusStream {

class CDriver : public CKernelDriverBase {
public:
    CDriver() : CKernelDriverBase("Census Stream") {}

    void Configure(const CDevice& xDevice, const SImageFormat& xFormat, const BlockMatcherCensus::SParameter& xPars,
                   int iDispDeltaThresh, EDataType eDispType = EDataType::UInt8) {
        detail::RequireInputFormat(xFormat, "CensusStream");
        detail::RequireDispConfig(xPars.xDispConfig, "CensusStream");
        if (!xPars.bLeftToRight) throw CError(CT_EINVAL, "CensusStream: the checked map is the left view's");
        EnsureHandle(ct_census_stream_create);
        const ct_format f = xFormat.ToC();
        const ct_census_match_params p{xPars.xDispConfig.iRange, xPars.iAggRadius, 1, xPars.xDispConfig.iMin};
        Ensure(ct_census_stream_configure(m_pHandle, xDevice.iDevice, &f, &p, iDispDeltaThresh,
                                          static_cast<int32_t>(eDispType)),
               "CensusStream::Configure");
    }

    /* Returns the frame number to Wait for. */
    int64_t Submit(const void* pLeft, size_t nLeftPitch, const void* pRight, size_t nRightPitch, void* pDisp,
                   size_t nDispPitch) {
        int64_t k = -1;
        Ensure(ct_census_stream_submit(m_pHandle, pLeft, nLeftPitch, pRight, nRightPitch, pDisp, nDispPitch, &k),
               "CensusStream::Submit");
        return k;
    }

    void Wait(int64_t iFrame) { Ensure(ct_census_stream_wait(m_pHandle, iFrame), "CensusStream::Wait"); }

    /* Device milliseconds from the next Submit's upload to the end of the
     * last download (TimerStop waits for every submitted frame). */
    void TimerStart() { Ensure(ct_census_stream_timer_start(m_pHandle), "CensusStream::TimerStart"); }
    float TimerStop() {
        float ms = 0.f;
        Ensure(ct_census_stream_timer_stop(m_pHandle, &ms), "CensusStream::TimerStop");
        return ms;
    }
};

}  // namespace CensusStream

/* Many pairs of mixed size per call: census both ways + cross-check. */
namespace BatchStereo {

struct SPair {
    _CDeviceSurface xImageL, xImageR, xDispChecked;
};

class CDriver : public CKernelDriverBase {
public:
    CDriver() : CKernelDriverBase("Batch Stereo") {}

    /* xFormats[i] / iDispRanges[i]: the shape of pair i. */
    void Configure(const CDevice& xDevice, const std::vector<SImageFormat>& xFormats,
                   const std::vector<int>& iDispRanges, int iDispDeltaThresh) {
        if (xFormats.size() != iDispRanges.size()) throw CError(CT_EINVAL, "BatchStereo: one range per format");
        std::vector<ct_batch_shape> shapes;
        for (size_t i = 0; i < xFormats.size(); ++i) {
            detail::RequireInputFormat(xFormats[i], "BatchStereo");
            shapes.push_back(ct_batch_shape{xFormats[i].iWidth, xFormats[i].iHeight, iDispRanges[i], 0});
        }
        EnsureHandle(ct_batch_create);
        Ensure(ct_batch_configure(m_pHandle, xDevice.iDevice, shapes.data(), int32_t(shapes.size()), iDispDeltaThresh),
               "BatchStereo::Configure");
    }

    void Process(const std::vector<SPair>& xPairs) {
        std::vector<ct_batch_item> items;
        for (const SPair& p : xPairs) {
            if (!p.xImageL.IsValid() || !p.xImageR.IsValid() || !p.xDispChecked.IsValid())
                throw CError(CT_EINVAL, "BatchStereo: empty surface in a pair");
            items.push_back(ct_batch_item{*p.xImageL.C(), *p.xImageR.C(), *p.xDispChecked.C()});
        }
        Ensure(ct_batch_process(m_pHandle, items.data(), int32_t(items.size()), S()), "BatchStereo::Process");
    }
};

}  // namespace BatchStereo

/* Learned confidence over census cost curves (D = 128): replaces the
 * right-to-left pass of the left-right check. */
namespace ConfidenceNet {

class CDriver : public CKernelDriverBase {
public:
    CDriver() : CKernelDriverBase("Confidence Net") {}

    void Configure(const CDevice& xDevice, int iMaxTrainBatch = 16) {
        EnsureHandle(ct_confnet_create);
        Ensure(ct_confnet_configure(m_pHandle, xDevice.iDevice, iMaxTrainBatch), "ConfidenceNet::Configure");
    }

    void SetParams(const std::vector<float>& params) {
        Ensure(ct_confnet_set_params(m_pHandle, params.data(), int32_t(params.size())), "ConfidenceNet::SetParams");
    }

    /* Raw little-endian fp32 weight file of CT_CONFNET_PARAMS floats. */
    void LoadParams(const std::string& path) {
        std::vector<float> p(CT_CONFNET_PARAMS);
        FILE* f = std::fopen(path.c_str(), "rb");
        if (!f) throw CError(CT_EINVAL, "ConfidenceNet::LoadParams: cannot open " + path);
        const size_t n = std::fread(p.data(), sizeof(float), p.size() + 1, f);
        std::fclose(f);
        if (n != p.size()) throw CError(CT_EINVAL, "ConfidenceNet::LoadParams: " + path + " is not a weight file");
        SetParams(p);
    }

    /* xScore (Single) and / or xDispChecked (the type of xDispLR): the
     * per-pixel score, and xDispLR with every disparity scoring below
     * fThreshold marked Inconsistent (UInt8: 255). */
    void Process(_CDeviceSurface& xScore, _CDeviceSurface& xDispChecked, const CCurveVolume& xCurves,
                 const _CDeviceSurface& xDispLR, float fThreshold) {
        Ensure(ct_confnet_infer(m_pHandle, xScore.C(), xCurves.C(), xDispLR.C(), xDispChecked.C(), fThreshold, S()),
               "ConfidenceNet::Process");
    }
};

}  // namespace ConfidenceNet

}  // namespace ctstereo

#endif  // CTSTEREO_HPP
