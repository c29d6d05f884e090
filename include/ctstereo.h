/*
 * ctstereo.h — C ABI of the ctstereo B200 stereo block-matching library.
 *
 * This boundary replaces the operator API of CluTec.Cuda's MultiView stereo
 * drivers. Each reference driver object
 *     CDriver::Configure(const CDevice&, const SImageFormat&, const SParameter&)
 *     CDriver::Process(output, left, right, ...)
 * becomes a handle with ct_<algo>_configure / ct_<algo>_process. Images are
 * caller-owned device buffers described by ct_image (the role of
 * _CDeviceSurface); parameters are plain structs passed to configure and used
 * as kernel arguments (the reference copies them into __constant__ symbols,
 * BlockMatcherNCC.cu:1393-1420); errors are int status codes instead of C++
 * exceptions (CLU_EXCEPTION / CLU_CUDA_ENSURE_OK, Api.cpp:86-95).
 *
 * Conventions
 *  - All process calls are asynchronous on the given stream and do no host
 *    synchronisation, except where stated (ct_crosscheck_range).
 *  - A handle may own device scratch (allocated in configure, freed by
 *    ct_destroy). It is not thread-safe: use one handle per host thread or
 *    lock externally; calls on one handle must not overlap on the GPU.
 *  - Disparity d in [disp_min, disp_min + D) maps a base pixel x to x - d in
 *    the other view for left-to-right matching and to x + d for right-to-left
 *    (the reference hides this in _SDisparityConfig::MapPixelPos, whose
 *    arithmetic is not available; this mapping is the library's definition).
 *    disp_min (the reference's xDispConfig.Min() / SAD1 iOffset) is 0 unless
 *    a matcher's parameters set it; maps hold the absolute disparity d.
 *  - Disparity map encodings:
 *      CT_PIX_U8 : d itself, 255 = not a disparity (invalid/inconsistent);
 *                  requires D <= 255.
 *      CT_PIX_U16: EDisparityId encoding (DisparityId.h:35-47): d + 1 for a
 *                  disparity (First = 1 .. Last = 0xFFEF), 0xFFFF
 *                  CannotEvaluate (window outside the image), 0xFFFA
 *                  Inconsistent (failed cross-check).
 *      CT_PIX_F32: sub-pixel disparity, -1.0f = invalid.
 */
#ifndef CTSTEREO_H
#define CTSTEREO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* cudaStream_t without including the CUDA headers. */
typedef struct CUstream_st* ct_stream;

/* ---- status codes ------------------------------------------------------ */
#define CT_OK 0
#define CT_EINVAL 1   /* bad argument: null pointer, size or parameter out of range */
#define CT_ETYPE 2    /* pixel type not supported ("Pixel types of given images not supported") */
#define CT_EFORMAT 3  /* image sizes disagree ("... do not have the same format") */
#define CT_ECUDA 4    /* a CUDA runtime call or kernel launch failed */
#define CT_ETIMEOUT 5 /* a bounded device-side wait gave up (status read back later) */
#define CT_ESTATE 6   /* handle of the wrong kind, or process before configure */
#define CT_ENOMEM 7   /* device allocation failed */
#define CT_EINTERNAL 8 /* a device-side consistency check failed (status read back later) */

/* ---- pixel types (TPixel_Lum_UInt8 etc.) -------------------------------- */
#define CT_PIX_U8 1
#define CT_PIX_U16 2
#define CT_PIX_U64 3
#define CT_PIX_F32 4
#define CT_PIX_RGBA8 5  /* 4 bytes per pixel: r, g, b, a (visualisation output) */
#define CT_PIX_F32X4 6  /* 16 bytes per pixel: 4 floats (3D map: x, y, z, valid) */
#define CT_PIX_U16X4 7  /* 8 bytes per pixel: 4 x uint16 (the reference matchers' TPixelEx output) */

/* EDisparityId codes used in CT_PIX_U16 maps (DisparityId.h:35-47). */
#define CT_DISP_FIRST 0x0001
#define CT_DISP_LAST 0xFFEF
#define CT_DISP_UNKNOWN 0x0000
#define CT_DISP_CANNOT_EVALUATE 0xFFFF
#define CT_DISP_SATURATED 0xFFFE
#define CT_DISP_NOT_FOUND 0xFFFD
#define CT_DISP_NOT_SPECIFIC 0xFFFC
#define CT_DISP_NOT_UNIQUE 0xFFFB
#define CT_DISP_INCONSISTENT 0xFFFA
#define CT_DISP_U8_INVALID 0xFF

/* A device image: the role of _CDeviceSurface (DeviceSurface.h:43-264), as a
 * pitched linear buffer instead of a cudaArray + surface object. */
typedef struct ct_image {
    void* ptr;            /* device pointer to row 0 */
    size_t pitch_bytes;   /* bytes between rows; >= width * element size */
    int32_t width;
    int32_t height;
    int32_t type;         /* CT_PIX_* */
    int32_t reserved;     /* must be 0 */
} ct_image;

/* Image format handed to configure: SImageFormat (width, height, pixel type). */
typedef struct ct_format {
    int32_t width;
    int32_t height;
    int32_t type;         /* pixel type of the input images: CT_PIX_U8 */
} ct_format;

typedef struct ct_handle ct_handle;

/* ---- common ------------------------------------------------------------ */

/* Message of the last failing call on this host thread ("" if none). */
const char* ct_last_error_string(void);
/* Library version, e.g. "ctstereo 0.1.0 sm_100a". */
const char* ct_version(void);
/* Release a handle of any kind and its device scratch. NULL is a no-op. */
int ct_destroy(ct_handle* h);
/* Device status word of the handle's last launches: 0 = fine, otherwise a
 * CT_E* code written by a kernel (a bounded wait gave up). Synchronises the
 * stream the handle last used, then clears the word. */
int ct_handle_device_status(ct_handle* h, int32_t* status);

/* ---- census transform: CensusTransform::CDriver -------------------------
 * Replaces CensusTransform.h:44-70 / CensusTransform.cu:60-157.
 *   CT_CENSUS_9X7: U8 -> U64. Window dx in [-4,4], dy in [-3,3]; the 63
 *     positions in raster order including the centre go to bits 62..0 (MSB
 *     first), bit 63 = 0; a bit is set iff neighbour > centre. Pixels within
 *     4 columns / 3 rows of the border get 0.
 *   CT_CENSUS_3X3: U8 -> U8, the reference transform exactly: 8 neighbours
 *     in raster order to bits 7..0, strict '>', 1-px border NOT written.
 */
#define CT_CENSUS_9X7 0
#define CT_CENSUS_3X3 1
typedef struct ct_census_params {
    int32_t window;       /* CT_CENSUS_9X7 or CT_CENSUS_3X3 */
} ct_census_params;

int ct_census_create(ct_handle** out);
/* CDriver::Configure(device, format) (CensusTransform.cu:125-135). */
int ct_census_configure(ct_handle* h, int32_t device, const ct_format* fmt, const ct_census_params* p);
/* CDriver::Process(trg, src) (CensusTransform.cu:138-157): src U8, dst U64
 * (9x7) or U8 (3x3), same width/height as configured. */
int ct_census_process(ct_handle* h, const ct_image* dst, const ct_image* src, ct_stream stream);
/* Both views of a stereo pair in one launch (CT_CENSUS_9X7 only): the same
 * result as two ct_census_process calls; the two outputs share one pitch. */
int ct_census_process_pair(ct_handle* h, const ct_image* dst_left, const ct_image* dst_right,
                           const ct_image* src_left, const ct_image* src_right, ct_stream stream);

/* ---- census block matcher -----------------------------------------------
 * 9x7 census of both images + Hamming cost (CensusDifference,
 * BlockMatcherNCC.cu:153-158, on 64-bit descriptors) + (2r+1)^2 box
 * aggregation + winner-take-all with the lowest d winning ties. A pixel is
 * valid iff its aggregation window is inside the image; disparity d is
 * searched iff the matched window is inside too. The handle owns the census
 * descriptor scratch (2 * W * H * 8 bytes) and a key buffer (W * H * 4).
 */
typedef struct ct_census_match_params {
    int32_t disp_count;     /* D, 1..256 */
    int32_t agg_radius;     /* r: 2 gives the 5x5 box (only 2 is built) */
    int32_t left_to_right;  /* 1: base = left image; 0: base = right image */
    int32_t disp_min;       /* xDispConfig.Min(): disparities disp_min .. disp_min + D - 1
                               (BlockMatcherNCC.cu:789-795); U8 maps need disp_min + D <= 255;
                               cost curves need 0 */
} ct_census_match_params;

int ct_bm_census_create(ct_handle** out);
int ct_bm_census_configure(ct_handle* h, int32_t device, const ct_format* fmt,
                           const ct_census_match_params* p);
/* disp: U8 or U16 W x H. left/right: U8 W x H. */
int ct_bm_census_process(ct_handle* h, const ct_image* disp, const ct_image* left,
                         const ct_image* right, ct_stream stream);
/* Both directions and the cross-check in one call: disp_lr / disp_rl (either
 * may be NULL when not wanted) receive the left-to-right and right-to-left
 * maps; disp_checked (may be NULL) the left map after the cross-check with
 * tolerance tol (CrossCheckDisparityMaps semantics). The left_to_right field
 * of the configured params is ignored here. */
int ct_bm_census_process_lr(ct_handle* h, const ct_image* disp_lr, const ct_image* disp_rl,
                            const ct_image* disp_checked, int32_t tol,
                            const ct_image* left, const ct_image* right, ct_stream stream);
/* Matching only, on census descriptors the caller computed with
 * ct_census_process (U64, CT_CENSUS_9X7): desc_base is the base view's
 * descriptors, desc_match the other view's; left_to_right selects x - d
 * (1) or x + d (0). Same output rules as ct_bm_census_process. */
int ct_bm_census_match_desc(ct_handle* h, const ct_image* disp, const ct_image* desc_base,
                            const ct_image* desc_match, int32_t left_to_right, ct_stream stream);

/* Cost-curve volume: the matcher's aggregated cost of every (pixel,
 * disparity), one byte each, the input of the learned confidence net
 * (ct_confnet_*). Code = 5x5 Hamming sum >> 3 (0..196); 255 for a disparity
 * whose match window leaves the image. Border pixels (within 2 of the image
 * edge) have no disparity and unspecified codes. Layout: groups g = 0 .. ceil(D/4) - 1
 * of 4 disparities; row (y, g) starts at ptr + (y * ceil(D/4) + g) *
 * pitch_bytes and holds one 32-bit word per pixel, word x + 2 for column x,
 * whose byte k (little-endian) is the code of disparity 4g + k. pitch_bytes
 * must be a multiple of 16 and at least 4 * (width + 2); ct_curves_pitch
 * gives the packed choice. No counterpart in the reference: its matchers
 * keep only the winning cost (BlockMatcherNCC.cu:491-592 WriteDisparity). */
typedef struct ct_curves {
    void* ptr;            /* device memory, 16-byte aligned, caller-owned */
    size_t pitch_bytes;
    int32_t width;
    int32_t height;
    int32_t disp_count;
    int32_t reserved;
} ct_curves;

/* Row pitch (bytes, a multiple of 256) of a curve volume of this width. */
int ct_curves_pitch(int32_t width, size_t* pitch_bytes);

/* ct_bm_census_process that also writes the cost-curve volume of the
 * configured direction (curves sized width x height x disp_count as
 * configured). The disparity map is identical to ct_bm_census_process. */
int ct_bm_census_process_curves(ct_handle* h, const ct_image* disp, const ct_curves* curves,
                                const ct_image* left, const ct_image* right, ct_stream stream);

/* Autotuner: times the kernel variants (4 or 8 disparities per warp) and
 * strip heights for this handle's (W, H, D, direction) on the given images,
 * keeps the fastest in the handle for later process calls. Synchronises
 * `stream`. (No counterpart in the reference, whose launch shapes are
 * compile-time SConfig constants, BlockMatcherNCC.h:43-79.) */
int ct_bm_census_autotune(ct_handle* h, const ct_image* left, const ct_image* right, ct_stream stream);
/* The handle's current launch shape (strip height in rows, disparities per
 * warp); either pointer may be NULL. */
int ct_bm_census_tuning(ct_handle* h, int32_t* strip_height, int32_t* disp_per_warp);
/* Sets the launch shape (e.g. from a saved tuning table): strip_height with
 * strip_height + 4 a multiple of 5 (11..511), disp_per_warp 4 or 8. Results do
 * not depend on it. */
int ct_bm_census_set_tuning(ct_handle* h, int32_t strip_height, int32_t disp_per_warp);
/* ct_bm_census_process_lr computes both directions in one matching pass by
 * default: the 5x5 Hamming cost of right pixel x_R at disparity e is the
 * left-to-right cost of left pixel x_R + e at e (the same two windows), so
 * the left-to-right pass also decides the right-to-left winners. enable = 0
 * selects two passes (one per direction, as the reference runs them); the
 * maps are identical either way. */
int ct_bm_census_set_fused_lr(ct_handle* h, int32_t enable);

/* Census matching that allocates nothing. No counterpart in the reference:
 * it exists for callers that cannot call cudaMalloc (a stream being captured
 * into a CUDA graph, a real-time loop with a frozen allocator, a host whose
 * device memory belongs to another framework's pool). Same kernels and
 * results as ct_bm_census_process with {disp_count, agg_radius 2,
 * left_to_right}, no handle; its scratch is a fixed static device array of
 * 40 MiB per GPU that loads the library, so images are limited to 2,097,152
 * pixels with rows rounded up to a multiple of 4 (1920 x 1080 fits; larger
 * -> CT_EINVAL).
 * Runs on the current device. Its first call on a device looks up the array
 * addresses: make it before any stream capture (the lookup is repeated when
 * the device's current context handle changes, e.g. after cudaDeviceReset).
 * Calls share the array, so calls that overlap on the GPU race; serialise
 * them. device_status (nullable, caller-owned device int32) receives
 * CT_ETIMEOUT if a bounded wait gives up; with NULL the code goes to a static
 * word that ct_bm_census_static_status reads. */
int ct_bm_census_process_static(const ct_image* disp, const ct_image* left, const ct_image* right,
                                int32_t disp_count, int32_t left_to_right, int32_t* device_status,
                                ct_stream stream);
/* Status word of the ct_bm_census_process_static calls on the current device
 * that passed no device_status: 0 = fine, else a CT_E* code. Synchronises the
 * device, then clears the word. Allocates nothing. */
int ct_bm_census_static_status(int32_t* status);

/* ---- SAD block matcher: BlockMatcherSAD1::CDriver ------------------------
 * Replaces BlockMatcherSAD1.h:42-127 / BlockMatcherSAD1.cu:493-596 for the
 * exhaustive mode: per-pixel |L - R| (EvalSAD, BlockMatcherSAD1.cu:151-153),
 * (2r+1)^2 box sum, winner-take-all over all D with lowest-d ties. (The
 * reference's coarse/fine search, gradient gate and SAD threshold are not
 * built; SAD1 is excluded from the reference's own build.)
 */
typedef struct ct_sad_params {
    int32_t disp_count;     /* iDispRange: D, 1..256 */
    int32_t radius;         /* EConfig patch: r = 4 gives 9x9; 1..4 */
    int32_t left_to_right;  /* 1: base = left image */
    int32_t disp_min;       /* iOffset: disparities disp_min .. disp_min + D - 1 */
} ct_sad_params;

int ct_bm_sad_create(ct_handle** out);
int ct_bm_sad_configure(ct_handle* h, int32_t device, const ct_format* fmt, const ct_sad_params* p);
/* CDriver::Process(disp, left, right): disp U8 or U16. */
int ct_bm_sad_process(ct_handle* h, const ct_image* disp, const ct_image* left,
                      const ct_image* right, ct_stream stream);

/* ---- NCC block matcher: BlockMatcherNCC::CDriver -------------------------
 * Replaces BlockMatcherNCC.h:41-144 / BlockMatcherNCC.cu:1270-1420.
 * Exact integer window sums (Sx, Sxx, Sy, Syy, Sxy) and FP32 normalisation:
 * ncc = float(n Sxy - Sx Sy) / sqrtf(float(n Sxx - Sx^2) * float(n Syy - Sy^2))
 * and 0 when sigma_x sigma_y < 1 (BlockMatcherNCC.cu:255-262). Argmax over d
 * with lowest-d ties. Left-to-right only. The score is not quantised.
 */
typedef struct ct_ncc_params {
    int32_t disp_count;     /* D, 1..256 */
    int32_t radius;         /* EConfig: 5 = Patch_11x11, 4 = Patch_9x9, 2 = Patch_5x5 */
    int32_t left_to_right;  /* must be 1 */
    int32_t disp_min;       /* xDispConfig.Min(): disparities disp_min .. disp_min + D - 1 */
} ct_ncc_params;

int ct_bm_ncc_create(ct_handle** out);
int ct_bm_ncc_configure(ct_handle* h, int32_t device, const ct_format* fmt, const ct_ncc_params* p);
/* disp U8/U16; score (nullable) F32 = NCC at the chosen d (0 for invalid
 * pixels). disp_init (nullable) switches on the guided mode
 * (MatcherUseDisparity, BlockMatcherNCC.cu:894-1255): a coarse disparity map
 * (U8 or U16 encoding) whose width divides the image width, s = width /
 * disp_init->width, with at least ceil(height / s) rows. Pixel (x, y) takes
 * the coarse disparity at (x / s, y / s) scaled by s; the pixels of each
 * 16 x 16 block (aligned to multiples of 16) search only
 * [max(0, min - 4), max + 4] of their block's scaled coarse disparities, and
 * get no disparity when none of them has one. */
int ct_bm_ncc_process(ct_handle* h, const ct_image* disp, const ct_image* score,
                      const ct_image* left, const ct_image* right, const ct_image* disp_init,
                      ct_stream stream);
/* enable = 1 (the default): unguided matching computes the window cross sums
 * on the tensor cores (tcgen05 MMAs on f16 pixels, exact fp32 sums); 0: on
 * the CUDA cores, as guided matching always does. Both give the same maps
 * and scores. */
int ct_bm_ncc_set_tensor_cores(ct_handle* h, int32_t enable);

/* ---- adaptive-window block matcher: BlockMatcherAW1 / AW2 ----------------
 * Replaces BlockMatcherAW1.h:41-157 and BlockMatcherAW2.h:41-135 with the
 * "best of 5 shifted windows" cost: A = min of the 7x7 SAD of the centred
 * window and of the windows shifted by +-3 px in x and in y; winner-take-all
 * (lowest d on ties) and FP32 parabolic sub-pixel refinement
 * d + (c- - c+) / (2 (c- - 2 c0 + c+)), skipped at d = 0, d = D-1 or when
 * d + 1 is not searchable. Left-to-right. Pixel valid iff 6 <= x < W-6 and
 * 6 <= y < H-6; d searched iff x - d - 6 >= 0.
 */
typedef struct ct_aw_params {
    int32_t disp_count;     /* D, 1..256 */
    int32_t left_to_right;  /* must be 1 */
    int32_t disp_min;       /* xDispConfig.Min(): disparities disp_min .. disp_min + D - 1 */
    int32_t reserved1;
} ct_aw_params;

int ct_bm_aw_create(ct_handle** out);
int ct_bm_aw_configure(ct_handle* h, int32_t device, const ct_format* fmt, const ct_aw_params* p);
/* disp: F32 (sub-pixel, -1 invalid) or U8/U16 (integer WTA). */
int ct_bm_aw_process(ct_handle* h, const ct_image* disp, const ct_image* left,
                     const ct_image* right, ct_stream stream);
/* Guided mode: CDriver::Process with xImageDispInit and iUseDispInput
 * (MatcherUseDisparity, BlockMatcherAW1.cu:996-1180). disp_init is a coarse
 * disparity map as for ct_bm_ncc_process; each 16 x 16 block takes its winner
 * over [max(0, min - 4), max + 4] of its scaled coarse disparities only (no
 * disparity when it has none); the sub-pixel step is unchanged. */
int ct_bm_aw_process_guided(ct_handle* h, const ct_image* disp, const ct_image* left,
                            const ct_image* right, const ct_image* disp_init, ct_stream stream);

/* ---- gradient gate of the plain matchers -----------------------------------
 * EvalGrad of the reference drivers (BlockMatcherSAD1.cu:226-249,
 * BlockMatcherNCC.cu:388-413, BlockMatcherAW1.cu:331-417): a pixel whose
 * patch has too little texture gets no disparity (U8 255, U16
 * CannotEvaluate, F32 -1; NCC score 0). SAD and NCC handles test the mean
 * |I(x) - I(x+1)| over the matching window (I = 0 beyond the right edge);
 * the AW handle tests the standard deviation over the 13 x 13 extent of its
 * five windows, truncated to an integer, in percent of 255. The base image
 * is the left one (the right one for right-to-left SAD). Applies to later
 * process calls; 0 (the default) switches it off. */
int ct_bm_set_gradient_gate(ct_handle* h, float grad_thresh);

/* ---- reference-compat output: the matchers' 4 x uint16 pixel ---------------
 * The reference matchers write TPixelEx = 4 x uint16 per pixel:
 *   x: disparity + EDisparityId::First, or Saturated (winner within the
 *      saturation band at the ends of the range), NotFound (score beyond the
 *      score threshold), NotSpecific (the scores next to the winner are within
 *      the minimum delta), CannotEvaluate (gradient gate, or the patch leaves
 *      the image), Unknown (no candidate);
 *   y: the winning score: SAD / N (SAD1, AW2), the NCC quantised to 0..255
 *      (NCC), or the similarity as a 16-bit percentage (AW1, BlockMatcher1);
 *   z, w: the specificity deltas before / after the winner, as the
 *      reference's sequential scan over the disparities records them.
 * Methods (each restates its driver, scan order and ID rules):
 *   CT_COMPAT_SAD1: BlockMatcherSAD1 (BlockMatcherSAD1.cu:279-488): P x P SAD
 *     (P = 3..16, Patch_16x16 centred at +8), scan from the largest disparity
 *     in steps of 4, then every disparity within 4 of the pixel's winner; a
 *     new minimum needs SAD / (P*P) < fSadThresh; z / w against the SAD before
 *     / after; Saturated for the 3 largest disparities; NotSpecific unless
 *     both deltas > iMinDeltaThresh. x holds the disparity + First (the
 *     reference's x holds the scan index + First).
 *   CT_COMPAT_NCC: BlockMatcherNCC (BlockMatcherNCC.cu:180-592): FP32 NCC
 *     from means and standard deviations, 0 when sigma_x sigma_y < 1,
 *     clamped at 0 and quantised to uint8; argmax ascending with the SSimStore
 *     bookkeeping; NotFound when max / 255 < fNccThresh; Saturated for the
 *     first 2 and the last disparity; NotSpecific unless both deltas >=
 *     iMinDeltaThresh. P = 5, 9, 11.
 *   CT_COMPAT_AW1: BlockMatcherAW1 (BlockMatcherAW1.cu:246-635): centre + best
 *     2 of 4 neighbouring s x s sub-windows (s = 3: Patch_9x9, 5:
 *     Patch_15x15, AdaptWnd_W32H16.h:240-285) of 255 - |a - b| (sim_type 0)
 *     or the signed product (1); thresholds fSimThresh and fMinDeltaThresh in
 *     percent.
 *   CT_COMPAT_AW2: BlockMatcherAW2 (BlockMatcherAW2.cu:143-382): centre + 2
 *     lowest of 4 sub-window SADs (AdaptWnd3D.h:244-300), scanned from the
 *     largest disparity; Saturated within 5 of the largest / 4 of the
 *     smallest scan index, as the reference compares them.
 *   CT_COMPAT_BM1: BlockMatcher1 (BlockMatcher1.cu:190-565): plain P x P
 *     window of (255 - |a - b|) >> 1 or the signed product x 127 (P = 5, 9,
 *     11, 15), thresholds as AW1.
 * Gates (grad_thresh > 0): mean |I(x) - I(x+1)| over the patch (SAD1, NCC),
 * the patch's standard deviation in percent (AW1 after truncation to an
 * integer, BM1), the AW2 neighbourhood over gradient sub-sums (AW2).
 * Divergences from the reference (its results there depend on its thread
 * tiling): a pixel is evaluated iff its patch is inside the image (else
 * (CannotEvaluate, 0, 0, 0)); a disparity is searched iff the matched patch
 * is inside; SAD1's fine pass is decided per pixel, not per thread block.
 */
#define CT_COMPAT_SAD1 0
#define CT_COMPAT_NCC 1
#define CT_COMPAT_AW1 2
#define CT_COMPAT_AW2 3
#define CT_COMPAT_BM1 4
typedef struct ct_compat_params {
    int32_t method;          /* CT_COMPAT_* */
    int32_t disp_count;      /* iDispRange / xDispConfig range: 1..256 */
    int32_t disp_min;        /* iOffset / xDispConfig.Min() */
    int32_t patch;           /* window side (SAD1, NCC, BM1) or sub-window side (AW1, AW2) */
    int32_t sim_type;        /* AW1, BM1: 0 absolute difference, 1 signed product */
    int32_t left_to_right;   /* 1: base = left, match x - d; 0: base = right, x + d */
    float grad_thresh;       /* fGradThresh (0: no gate) */
    float score_thresh;      /* fSadThresh / fNccThresh / fSimThresh */
    float min_delta_thresh;  /* iMinDeltaThresh (integer part; SAD1, NCC, AW2) / fMinDeltaThresh (AW1, BM1) */
    int32_t reserved[3];     /* 0 */
} ct_compat_params;

int ct_bm_compat_create(ct_handle** out);
/* CDriver::Configure of the chosen reference driver. */
int ct_bm_compat_configure(ct_handle* h, int32_t device, const ct_format* fmt, const ct_compat_params* p);
/* CDriver::Process(disp, left, right): disp CT_PIX_U16X4 (all four channels)
 * or CT_PIX_U16 (the x channel only); left / right U8. */
int ct_bm_compat_process(ct_handle* h, const ct_image* disp, const ct_image* left, const ct_image* right,
                         ct_stream stream);

/* ---- cross-check: CrossCheckDisparityMaps::CDriver ------------------------
 * Replaces CrossCheckDisparityMaps.h:38-117 / .cu:63-190, with the
 * reference kernel's rule exactly. For each pixel of disp_base inside the
 * 1-pixel image frame holding a disparity code v = d + First: x' = x - d
 * (left_to_right = 1) or x + d; if x' is outside the image, or
 * |disp_other(x') - v| > disp_delta_thresh with disp_other's code compared
 * raw (an ID or Unknown there is compared by its value, as the reference
 * does), the result is Inconsistent; otherwise v is kept. Non-disparity
 * inputs are copied through. The frame pixels of result are not written, as
 * in the reference. U8 maps (255 = not a disparity; no reference
 * counterpart) keep d only against a disparity within the tolerance. The
 * min / max of the kept disparities is reduced on the device (the reference
 * does a per-thread atomic range plus two blocking copies and a host
 * reduction).
 */
typedef struct ct_crosscheck_params {
    int32_t disp_delta_thresh;  /* iDispDeltaThresh */
    int32_t left_to_right;      /* iIsLeftToRight */
    int32_t reserved0;
    int32_t reserved1;
} ct_crosscheck_params;

int ct_crosscheck_create(ct_handle** out);
int ct_crosscheck_configure(ct_handle* h, int32_t device, const ct_format* fmt,
                            const ct_crosscheck_params* p);
/* result, disp_base, disp_other: same size and type (U8 or U16). */
int ct_crosscheck_process(ct_handle* h, const ct_image* result, const ct_image* disp_base,
                          const ct_image* disp_other, ct_stream stream);
/* CDriver::DispMin() / DispMax(): synchronises the last process stream and
 * returns the kept range in disparity units (min > max when none kept). */
int ct_crosscheck_range(ct_handle* h, int32_t* disp_min, int32_t* disp_max);

/* ---- batched census stereo ------------------------------------------------
 * Many pairs of mixed size and disparity range per call: 9x7 census of both
 * images, census matching in both directions (one fused pass per pair that
 * decides both directions' winners), cross-check with tolerance tol, for
 * every pair. One batched census launch and one persistent,
 * work-queue-scheduled matching launch (one CTA per SM) whose last CTAs per
 * strip run the cross-check. Each pair's result equals
 * ct_bm_census_process_lr(disp_checked) run on that pair alone. No
 * counterpart in the reference (its drivers process one image per call).
 * The handle owns all scratch; pair shapes are fixed at configure. The
 * scratch's counters and right-view keys return to their initial state at
 * the end of every complete call; after a call whose status word reports
 * CT_ETIMEOUT, configure the handle again before the next call. */
typedef struct ct_batch_shape {
    int32_t width;
    int32_t height;
    int32_t disp_count;   /* 1..256 */
    int32_t reserved;
} ct_batch_shape;

typedef struct ct_batch_item {
    ct_image left;        /* U8 */
    ct_image right;       /* U8 */
    ct_image disp;        /* U8 (disp_count <= 255) or U16: the cross-checked left map */
} ct_batch_item;

int ct_batch_create(ct_handle** out);
/* Up to 256 pairs; strip heights start from a cost model per (W, H, D). */
int ct_batch_configure(ct_handle* h, int32_t device, const ct_batch_shape* shapes, int32_t n, int32_t tol);
/* items[i] must match shapes[i]. Asynchronous on stream, except that it
 * first waits for this handle's previous call (its pinned staging buffer is
 * reused). */
int ct_batch_process(ct_handle* h, const ct_batch_item* items, int32_t n, ct_stream stream);
/* Autotuner: times the whole batch on these items for candidate strip heights
 * of each distinct (W, H, D) and keeps the fastest. Synchronises stream. */
int ct_batch_autotune(ct_handle* h, const ct_batch_item* items, int32_t n, ct_stream stream);
/* Strip height chosen for pair `pair` (index into the configured shapes). */
int ct_batch_strip_height(ct_handle* h, int32_t pair, int32_t* strip_height);
/* Captures one process call on these items into a CUDA graph held by the
 * handle (the items' buffers must stay valid); ct_batch_graph_launch replays
 * it on any stream without host work. Re-configure or autotune drops it. */
int ct_batch_graph_create(ct_handle* h, const ct_batch_item* items, int32_t n);
int ct_batch_graph_launch(ct_handle* h, ct_stream stream);

/* ---- streamed census stereo ----------------------------------------------
 * Frames in host memory in, cross-checked maps in host memory out, with the
 * upload of one frame and the download of another overlapping the matching
 * of a third (three device slots; copies and matching on three internal
 * streams ordered by events). Each frame's map equals
 * ct_bm_census_process_lr(disp_checked) on that pair. No counterpart in the
 * reference (its CDeviceSurface::CopyFrom / CopyInto are synchronous copies
 * around a blocking Process). Host images are rows of `pitch` bytes;
 * page-locked memory (cudaHostAlloc / cudaHostRegister) lets the copies run
 * behind the matching, pageable memory works but serialises frames. */
int ct_census_stream_create(ct_handle** out);
/* fmt: the pair's format (U8); p: the census matcher parameters (D, radius 2);
 * tol: cross-check tolerance; out_type: CT_PIX_U8 or CT_PIX_U16 maps. */
int ct_census_stream_configure(ct_handle* h, int32_t device, const ct_format* fmt,
                               const ct_census_match_params* p, int32_t tol, int32_t out_type);
/* Enqueues one frame and returns at once with its number in *frame. left,
 * right and checked must stay valid, and left / right unchanged, until
 * ct_census_stream_wait for that frame has returned. */
int ct_census_stream_submit(ct_handle* h, const void* left, size_t left_pitch, const void* right,
                            size_t right_pitch, void* checked, size_t checked_pitch, int64_t* frame);
/* Blocks until the frame's map is in host memory (also reports a device
 * status word set by the matching, as CT_ETIMEOUT / CT_EINTERNAL). */
int ct_census_stream_wait(ct_handle* h, int64_t frame);
/* Device time of a run of frames: start marks the point before the next
 * frame's upload; stop waits for every submitted frame and returns the
 * milliseconds from the mark to the end of the last download. */
int ct_census_stream_timer_start(ct_handle* h);
int ct_census_stream_timer_stop(ct_handle* h, float* ms);

/* ---- disparity visualisation: ColorDisparityImage::CDriver -----------------
 * Replaces ColorDisparityImage.h:37-120 / ColorDisparityImage.cu:45-300,
 * writing a headless device image instead of a GL surface. disp: U16
 * (EDisparityId codes) or U8 (d, read as code d + 1; 255 as CannotEvaluate).
 * t = (code - disp_min) / (disp_max - disp_min) in FP32, q(t, M) =
 * rint(clamp(t, 0, 1) * M). Styles (EStyle):
 *   CT_COLOR_ANALYSIS  out RGBA8: disparities gray q(t, 255); each other code
 *                      its colour from `colors` (unknown codes: red)
 *   CT_COLOR_GRAY      out U16: disparities q(t, 65535), others 0
 *   CT_COLOR_COLOR     out RGBA8: the blue-green-red ramp of NormFloatToColor
 *                      (Conversion.h:56-74), others black
 *   CT_COLOR_DISP_ABS  out U16: disparities their code, others 0
 *   CT_COLOR_DISP_REL  out U16: (0x7FFF + inf_offset) - (code - 1), others 0
 * Colours are RGBA8 words with r in the low byte, in the order unknown,
 * cannot evaluate, saturated, not specific, not found, not unique,
 * inconsistent. disp_min / disp_max are codes (d + 1). */
#define CT_COLOR_ANALYSIS 0
#define CT_COLOR_GRAY 1
#define CT_COLOR_COLOR 2
#define CT_COLOR_DISP_ABS 3
#define CT_COLOR_DISP_REL 4
typedef struct ct_color_params {
    int32_t style;        /* CT_COLOR_* */
    int32_t disp_min;     /* uDispMin (code) */
    int32_t disp_max;     /* uDispMax (code) */
    int32_t inf_offset;   /* uDispInfOffset (DISP_REL) */
    uint32_t colors[7];   /* pixUnknown .. pixInconsistent */
} ct_color_params;

/* SParameter's defaults (ColorDisparityImage.h:75-87): range First .. Last,
 * the reference's ID colours. */
int ct_color_params_default(int32_t style, ct_color_params* p);
/* CDriver::Process(color image, disparity image, style); asynchronous. */
int ct_color_disparity(const ct_image* out, const ct_image* disp, const ct_color_params* p, ct_stream stream);

/* ---- disparity mip-maps: CreateDispMipMaps::CDriver ------------------------
 * Replaces CreateDispMipMaps.h:44-80 / CreateDispMipMaps.cu:66-330 and the
 * packed mip-map surface _CDeviceSurfMipMap / CDeviceSurfMipMap
 * (DeviceSurfMipMap.h:40-150, DeviceSurfMipMap.cpp:68-146). One F32 image
 * holds every level: level 0 (W x H) at (0, 0), level k >= 1 at
 * (X1, H_1 + ... + H_{k-1}) with X1 = W rounded up to a multiple of 4,
 * W_{k+1} = (W_k - 1) / 2 and H_{k+1} = (H_k - 1) / 2; the image is
 * (X1 + (W - 1) / 2) x H. Level 0 = the codes as floats (First .. Last ->
 * the code, other IDs -> 0 = Unknown; U8 maps are read as code d + 1, 255 as
 * CannotEvaluate); level k + 1 = the 1-2-1 weighted mean of the non-zero
 * entries of level k horizontally at x = 2i .. 2i + 2, then vertically at
 * y = 2j .. 2j + 2, times 0.5 (SmoothHorizontalLum / SmoothVerticalLum,
 * bit-identical, IEEE division). */

/* Packed image width for a width x height disparity map (its height is
 * height) and the maximal level count (CDeviceSurfMipMap::Create and
 * MaxMipMapLevelCount; the number of levels k >= 1 that are not empty). */
int ct_disp_mipmap_format(int32_t width, int32_t height, int32_t* packed_width, int32_t* max_levels);
/* Origin and size of level 0 .. max_levels in the packed image
 * (_CDeviceSurfMipMap::GetOrigin / Format). Every origin is 16-byte aligned
 * in a 16-byte aligned image, so a level can be passed on as a ct_image. */
int ct_disp_mipmap_level(int32_t width, int32_t height, int32_t level, int32_t* x, int32_t* y, int32_t* w,
                         int32_t* h);
/* CDriver::Run(mip-map, temp, disparity, level_count): writes levels
 * 0 .. level_count - 1 of `mipmap` (F32, the packed size) from disp (U16 or
 * U8). As in the reference, level_count > max_levels is CT_EINVAL,
 * level_count <= 0 means max_levels, and level_count == 1 writes nothing.
 * Asynchronous; no scratch memory. */
int ct_disp_mipmaps(const ct_image* mipmap, const ct_image* disp, int32_t level_count, ct_stream stream);

/* ---- learned confidence ------------------------------------------------------
 * A small network that scores, per pixel, how likely the census matcher's
 * winner-take-all disparity is correct, from the pixel's cost curve
 * (ct_curves, D = 128). It stands in for the right-to-left pass of the
 * left-right check (CrossCheckDisparityMaps.cu:63-110), which stays the
 * fallback and the yardstick for its error. No counterpart in the reference.
 *
 * Input: the pixel's curve re-centred on its winning disparity d (taken from
 * the left-to-right disparity map): sample r[k] = c[d - 64 + k], 255 outside
 * the curve; the convolutions read its 35 central codes r[52 .. 86] (the
 * disparities d - 12 .. d + 22).
 * Network: conv1 1->32 (k=5, stride 5) -> ReLU -> conv2 32->32 (k=5, stride
 * 3, pad 1) -> ReLU -> conv3 32->32 (k=5, pad 2, one output) -> ReLU -> fc1
 * 32->64 -> ReLU -> fc2 64->1 -> sigmoid. Weights bf16
 * (fp32 master copies during training), biases fp32, accumulation fp32, conv
 * activations rounded to bf16. Flat parameter order (CT_CONFNET_PARAMS
 * floats): w1[32][5], b1[32], w2[32][32][5] ([out][in][tap]), b2[32],
 * w3[32][32][5], b3[32], w4[64][32], b4[64], w5[64], b5.
 *
 * Training runs on the GPU with the library's own forward/backward kernels
 * (CUDA cores, fp32 accumulation) and Adam; inference over a whole curve
 * volume runs on the tensor cores (tcgen05, fp32 accumulation in TMEM).
 * Device pointers below (samples, labels, xy, grad, loss, scores) are device
 * memory. */
#define CT_CONFNET_PARAMS 12673

int ct_confnet_create(ct_handle** out);
/* Allocates training scratch for up to max_batch samples per step and
 * initialises the weights (ct_confnet_init with seed 1). */
int ct_confnet_configure(ct_handle* h, int32_t device, int32_t max_batch);
/* He-style random initialisation from a seed; resets the optimiser. */
int ct_confnet_init(ct_handle* h, uint64_t seed);
/* Host fp32 parameter vectors (save / load); set resets the optimiser. */
int ct_confnet_set_params(ct_handle* h, const float* params, int32_t n);
int ct_confnet_get_params(ct_handle* h, float* params, int32_t n);
/* samples[n][128] (bytes) = re-centred curves at pixels xy[n] = (x, y)
 * pairs; disp (U8 or U16, same size as the curves) holds the winners. */
int ct_confnet_gather(ct_handle* h, uint8_t* samples, const ct_curves* curves, const ct_image* disp,
                      const int32_t* xy, int32_t n, ct_stream stream);
/* Mean binary cross-entropy of n samples (labels: 1 = disparity correct)
 * and its gradient (CT_CONFNET_PARAMS floats); either output may be NULL. */
int ct_confnet_loss_grad(ct_handle* h, const uint8_t* samples, const uint8_t* labels, int32_t n, float* grad,
                         float* loss, ct_stream stream);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on n samples; loss may be NULL. */
int ct_confnet_train_step(ct_handle* h, const uint8_t* samples, const uint8_t* labels, int32_t n, float lr,
                          float* loss, ct_stream stream);
/* Scores (sigmoid) of n samples through the training forward. */
int ct_confnet_scores(ct_handle* h, float* scores, const uint8_t* samples, int32_t n, ct_stream stream);
/* Scores of a whole curve volume on the tensor cores. disp: the
 * left-to-right winner map (U8 or U16) the curves came with. Outputs (either
 * may be NULL, not both): score (F32, P(disparity correct) per pixel) and
 * checked (same type as disp): disp with every disparity whose score is
 * below threshold marked invalid, in the encoding the cross-check uses
 * (U16 CT_DISP_INCONSISTENT, U8 255), so it replaces disp_checked of
 * ct_bm_census_process_lr. The first call after new weights packs them
 * (synchronises the previous stream). */
int ct_confnet_infer(ct_handle* h, const ct_image* score, const ct_curves* curves, const ct_image* disp,
                     const ct_image* checked, float threshold, ct_stream stream);

/* ---- disparity to 3D: MapDisparityTo3D::CDriver ---------------------------
 * Replaces MapDisparityTo3D.h:41-150 / MapDisparityTo3D.cu:75-330. The
 * reference's stereo camera (Clu::Camera::_CStereoPinhole, CluTec.Core, not in
 * the reference tree) is replaced by two explicit pinhole cameras: pixel
 * (x, y) of a camera looks along R ((x - cx) / fx, (y - cy) / fy, 1) from its
 * centre (camera axes x right, y down, z forward; R = camera-to-world
 * rotation, row-major). For each pixel of the left disparity map: code c
 * (U16 as stored; U8 d read as d + 1, 255 as CannotEvaluate; F32 sub-pixel
 * d >= 0 read as d + 1, negative as CannotEvaluate) is valid if disp_min <=
 * c <= disp_max; the disparity is c - 1 if valid, else disp_min (as the
 * reference, MapDisparityTo3D.cu:111-121); the left ray through (x, y) and
 * the right ray through (x - d, y) are intersected at the midpoint of their
 * closest points. Output (F32X4): (X, Y, Z, valid) in world coordinates, with
 * Y and Z negated when cs_rut = 1 (x right, y up, z towards, the reference's
 * bIsCsRUT); (0, 0, 0, 0) where the rays are parallel. The range of the
 * valid intersected points is reduced on the device (ct_map3d_range). */
typedef struct ct_pinhole {
    float fx, fy;       /* focal lengths in pixels */
    float cx, cy;       /* principal point in pixels */
    float rot[9];       /* camera-to-world rotation, row-major */
    float center[3];    /* projection centre in world coordinates */
} ct_pinhole;

typedef struct ct_map3d_params {
    int32_t disp_min, disp_max;  /* valid codes (uDispMin, uDispMax) */
    int32_t cs_rut;              /* bIsCsRUT */
    int32_t reserved;            /* 0 */
    ct_pinhole cam[2];           /* left, right (camStereoPinhole) */
} ct_map3d_params;

int ct_map3d_create(ct_handle** out);
/* CDriver::Configure(device, format, parameters); format = the disparity
 * map's size and type (U8, U16 or F32). */
int ct_map3d_configure(ct_handle* h, int32_t device, const ct_format* fmt, const ct_map3d_params* p);
/* CDriver::Process(3D map, disparity map): map3d F32X4, same size. */
int ct_map3d_process(ct_handle* h, const ct_image* map3d, const ct_image* disp, ct_stream stream);
/* pixMin / pixMax of the last process call (x, y, z of the valid intersected
 * points; FLT_MAX / -FLT_MAX when there were none). Synchronises. */
int ct_map3d_range(ct_handle* h, float* min_xyz, float* max_xyz);

/* ---- pipe-rate probe ---------------------------------------------------------
 * Measures the issue rate of the integer operations the matchers are built
 * from on the given device (a few ms of GPU time), as operations per SM per
 * clock, plus the SM clock seen. Used for the integer-pipe roofline. */
typedef struct ct_pipe_rates {
    double popc_per_clk_sm;     /* 32-bit POPC */
    double iadd3_per_clk_sm;    /* IADD3 */
    double lop3_per_clk_sm;     /* LOP3 (xor) */
    double vimnmx_per_clk_sm;   /* packed u16x2 3-way min */
    double imad_per_clk_sm;     /* IMAD */
    double sm_clock_mhz;        /* clock measured during the probe */
    int32_t sm_count;
    int32_t reserved;
} ct_pipe_rates;
int ct_probe_pipe_rates(int32_t device, ct_pipe_rates* out);

/* Self-test of the failure reporting of bounded device waits (the reference
 * has none: its kernels do not wait on each other). Launches one CTA on the
 * handle's device that waits on an mbarrier nothing ever arrives at, with a
 * limit of poll_limit polls (1 .. 1048576), through the same bounded wait the
 * TMA consumers use. The wait gives up and writes CT_ETIMEOUT into the
 * handle's device status word, which ct_handle_device_status then returns,
 * as it would for a tile that never arrived; the kernel returns normally and
 * the context stays usable. The handle must be configured. */
int ct_handle_test_wait_timeout(ct_handle* h, uint32_t poll_limit, ct_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* CTSTEREO_H */
