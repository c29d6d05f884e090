/*
 * ctsynth.h — C ABI of libctsynth.so, the seeded synthetic stereo-pair
 * generator that the tests, the benchmark and the confidence-net trainer use
 * for inputs with ground truth. It is a separate host-only library, not part
 * of the matcher library (libctstereo.so), so a CPU run that only needs
 * inputs loads no matcher code. No counterpart in the reference, whose demo
 * reads a stereo pair from disk (UsertTest1.cpp:59-61).
 * Returns CT_OK or CT_EINVAL (codes of ctstereo.h).
 */
#ifndef CTSYNTH_H
#define CTSYNTH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- synthetic stereo pairs -----------------------------------------------
 * Seeded generator of rectified stereo pairs with ground truth (host memory).
 *   kind 1: fractal value noise (4 octaves) left image; disparity = 4
 *           background + 8 fronto-parallel rectangles in [0, dmax]; right =
 *           forward warp with occlusion handling + N(0, 2^2); disoccluded
 *           right pixels get fresh noise.
 *   kind 2: 24 slanted planes (|grad d| <= 0.1 px/px, rounded), noise 3.
 *   kind 3: 6 smooth Gaussians scaled to [0, dmax] + 12 sharp rectangles,
 *           right-image gain in [0.9, 1.1], noise 2.
 * gt: int16 left-view ground truth disparity; occ: 1 where the left pixel is
 * occluded in the right view (or maps outside it). Any output may be NULL.
 */
int ct_synth_pair(int32_t kind, uint64_t seed, int32_t width, int32_t height, int32_t dmax,
                  uint8_t* left, uint8_t* right, int16_t* gt, uint8_t* occ);

#ifdef __cplusplus
}
#endif
#endif /* CTSYNTH_H */
