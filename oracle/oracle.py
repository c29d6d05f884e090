"""ctypes loader for the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference legs of bench.py as the checker. The product code
never imports this module.

Every function takes and returns numpy arrays; disparities are int16 with -1
for invalid pixels (and -2 for cross-check failures).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

_DIR = Path(__file__).resolve().parent
LIB_PATH = _DIR / "liboracle.so"
_lib = None


def build() -> Path:
    """Builds liboracle.so with the Makefile next to this file."""
    subprocess.run(["make", "-s", "-C", str(_DIR)], check=True)
    return LIB_PATH


def use_native() -> str:
    """Switches this process to liboracle_native.so, compiled here with
    -march=native for the host's own cores (the CPU-baseline timing). Must run
    before the first lib() call; falls back to the portable x86-64-v3 build if
    the compiler fails. Returns the -march used."""
    global LIB_PATH
    if _lib is not None:
        return "native" if LIB_PATH.name == "liboracle_native.so" else "x86-64-v3"
    # always rebuilt (-B): a copy built on another host may use instructions this one lacks
    r = subprocess.run(["make", "-B", "-s", "-C", str(_DIR), "native"], capture_output=True, text=True)
    if r.returncode == 0 and (_DIR / "liboracle_native.so").exists():
        LIB_PATH = _DIR / "liboracle_native.so"
        return "native"
    return "x86-64-v3"


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(LIB_PATH))
        vp, i = C.c_void_p, C.c_int
        _lib.or_num_threads.restype = i
        _lib.or_set_threads.argtypes = [i]
        _lib.or_census3x3.argtypes = [vp, i, i, i, vp, i]
        _lib.or_census9x7.argtypes = [vp, i, i, i, vp, i]
        _lib.or_match_census_desc.argtypes = [vp, vp, i, i, i, i, i, i, vp, vp, vp, i]
        _lib.or_match_census.argtypes = [vp, vp, i, i, i, i, i, i, i, vp, vp, vp, i]
        _lib.or_match_sad.argtypes = [vp, vp, i, i, i, i, i, i, i, vp, vp]
        _lib.or_match_aw.argtypes = [vp, vp, i, i, i, i, i, vp, vp, vp, vp]
        _lib.or_match_aw_guided.argtypes = [vp, vp, i, i, i, i, i, vp, vp, vp, vp, vp, vp]
        _lib.or_match_ncc.argtypes = [vp, vp, i, i, i, i, i, i, vp, vp, vp]
        _lib.or_match_ncc_guided.argtypes = [vp, vp, i, i, i, i, i, i, vp, vp, vp, vp, vp]
        _lib.or_crosscheck.argtypes = [vp, vp, i, i, i, i, vp, vp]
        _lib.or_crosscheck_codes.argtypes = [vp, vp, i, i, i, i, i, vp, vp]
        _lib.or_box_sums.argtypes = [vp, i, i, i, i, vp]
        _lib.or_div_int_mismatches.argtypes = [i, i]
        _lib.or_div_int_mismatches.restype = C.c_long
        f = C.c_float
        _lib.or_compat_match.argtypes = [vp, vp, i, i, i, i, i, i, i, i, i, f, f, f, vp]
        _lib.or_gate_mask.argtypes = [vp, i, i, i, i, i, f, vp]
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data)


def _u8(a):
    a = np.ascontiguousarray(a, dtype=np.uint8)
    assert a.ndim == 2
    return a


def num_threads() -> int:
    return lib().or_num_threads()


def set_threads(n: int) -> None:
    lib().or_set_threads(n)


def census9x7(img):
    img = _u8(img)
    H, W = img.shape
    out = np.empty((H, W), np.uint64)
    lib().or_census9x7(_p(img), W, H, W, _p(out), W)
    return out


def census3x3(img, fill=0):
    img = _u8(img)
    H, W = img.shape
    out = np.full((H, W), fill, np.uint8)
    lib().or_census3x3(_p(img), W, H, W, _p(out), W)
    return out


def match_census(L, R, D, r=2, left_to_right=True, curve_shift=None, dmin=0):
    """Disparities dmin .. dmin + D - 1 -> (disp int16, best cost int32[,
    curve uint8 HxWxD indexed by disparity - dmin])"""
    L, R = _u8(L), _u8(R)
    H, W = L.shape
    disp = np.empty((H, W), np.int16)
    cost = np.empty((H, W), np.int32)
    curve = None
    if curve_shift is not None:
        curve = np.full((H, W, D), 255, np.uint8)
    lib().or_match_census(_p(L), _p(R), W, H, W, D, dmin, r, 0 if left_to_right else 1, _p(disp), _p(cost),
                          _p(curve) if curve is not None else None, curve_shift or 0)
    return (disp, cost) if curve is None else (disp, cost, curve)


def match_census_desc(cb, cm, D, r=2, left_to_right=True, dmin=0):
    cb = np.ascontiguousarray(cb, np.uint64)
    cm = np.ascontiguousarray(cm, np.uint64)
    H, W = cb.shape
    disp = np.empty((H, W), np.int16)
    cost = np.empty((H, W), np.int32)
    lib().or_match_census_desc(_p(cb), _p(cm), W, H, D, dmin, r, 0 if left_to_right else 1, _p(disp), _p(cost),
                               None, 0)
    return disp, cost


def match_sad(L, R, D, r=4, left_to_right=True, dmin=0):
    L, R = _u8(L), _u8(R)
    H, W = L.shape
    disp = np.empty((H, W), np.int16)
    cost = np.empty((H, W), np.int32)
    lib().or_match_sad(_p(L), _p(R), W, H, W, D, dmin, r, 0 if left_to_right else 1, _p(disp), _p(cost))
    return disp, cost


def match_aw(L, R, D, dmin=0):
    """-> (disp int16, cost int32, sub32 float32, sub64 float64)"""
    L, R = _u8(L), _u8(R)
    H, W = L.shape
    disp = np.empty((H, W), np.int16)
    cost = np.empty((H, W), np.int32)
    s32 = np.empty((H, W), np.float32)
    s64 = np.empty((H, W), np.float64)
    lib().or_match_aw(_p(L), _p(R), W, H, W, D, dmin, _p(disp), _p(cost), _p(s32), _p(s64))
    return disp, cost, s32, s64


def match_aw_guided(L, R, D, coarse, dmin=0):
    """Guided adaptive-window matcher (see guide_ranges) -> as match_aw."""
    L, R = _u8(L), _u8(R)
    H, W = L.shape
    lo, hi = guide_ranges(coarse, W, H)
    disp = np.empty((H, W), np.int16)
    cost = np.empty((H, W), np.int32)
    s32 = np.empty((H, W), np.float32)
    s64 = np.empty((H, W), np.float64)
    lib().or_match_aw_guided(_p(L), _p(R), W, H, W, D, dmin, _p(lo), _p(hi), _p(disp), _p(cost), _p(s32),
                             _p(s64))
    return disp, cost, s32, s64


def match_ncc(L, R, D, r=5, dmin=0):
    """-> (disp int16, score32 float32, score64 float64)"""
    L, R = _u8(L), _u8(R)
    H, W = L.shape
    disp = np.empty((H, W), np.int16)
    s32 = np.empty((H, W), np.float32)
    s64 = np.empty((H, W), np.float64)
    lib().or_match_ncc(_p(L), _p(R), W, H, W, D, dmin, r, _p(disp), _p(s32), _p(s64))
    return disp, s32, s64


GUIDE_BLOCK = 16   # pixels per side of a guide group
GUIDE_MARGIN = 4   # disparities searched below / above the group's coarse range


def guide_ranges(coarse, W, H):
    """Search ranges of the guided mode (MatcherUseDisparity,
    BlockMatcherNCC.cu:980-1168), per pixel: coarse is an int16 disparity map
    (-1 = no disparity) with W / coarse.shape[1] = s an integer. Pixel (x, y)
    reads the coarse disparity at (x // s, y // s), scaled by s; the pixels of
    each 16 x 16 block (blocks aligned to multiples of 16) share the range
    [max(0, min - 4), max + 4] of their block's scaled coarse disparities, or
    no range (lo > hi) when the block has none. -> (lo, hi) int32 (H, W)."""
    coarse = np.asarray(coarse, np.int16)
    Hc, Wc = coarse.shape
    s = W // Wc
    assert s * Wc == W and -(-H // s) <= Hc
    ys, xs = np.arange(H) // s, np.arange(W) // s
    up = coarse[ys][:, xs].astype(np.int64)
    up = np.where(up >= 0, up * s, -1)
    B = GUIDE_BLOCK
    gh, gw = -(-H // B), -(-W // B)
    lo = np.full((gh, gw), 1 << 20, np.int64)
    hi = np.full((gh, gw), -1, np.int64)
    for gy in range(gh):
        for gx in range(gw):
            blk = up[gy * B:(gy + 1) * B, gx * B:(gx + 1) * B]
            v = blk[blk >= 0]
            if v.size:
                lo[gy, gx] = max(0, int(v.min()) - GUIDE_MARGIN)
                hi[gy, gx] = int(v.max()) + GUIDE_MARGIN
    return (np.ascontiguousarray(np.repeat(np.repeat(lo, B, 0), B, 1)[:H, :W], np.int32),
            np.ascontiguousarray(np.repeat(np.repeat(hi, B, 0), B, 1)[:H, :W], np.int32))


def match_ncc_guided(L, R, D, coarse, r=5, dmin=0):
    """Guided NCC (see guide_ranges) -> (disp int16, score32, score64)."""
    L, R = _u8(L), _u8(R)
    H, W = L.shape
    lo, hi = guide_ranges(coarse, W, H)
    disp = np.empty((H, W), np.int16)
    s32 = np.empty((H, W), np.float32)
    s64 = np.empty((H, W), np.float64)
    lib().or_match_ncc_guided(_p(L), _p(R), W, H, W, D, dmin, r, _p(lo), _p(hi), _p(disp), _p(s32), _p(s64))
    return disp, s32, s64


def color_disparity(codes, style, disp_min=1, disp_max=0xFFEF, inf_offset=0, colors=None):
    """Disparity visualisation (ColorDisparityImage.cu:45-300; the ramp of
    NormFloatToColor, Conversion.h:56-74) on a U16 EDisparityId code map.
    RGBA8 styles return uint32 words (r in the low byte), the others uint16.
    NormFloatTo (CluTec.Core, not in the reference tree) is restated as
    rint(clamp(t, 0, 1) * max)."""
    f32 = np.float32
    c = np.asarray(codes).astype(np.int64)
    disp = (c >= 1) & (c <= 0xFFEF)
    t = (c - disp_min).astype(f32) / f32(disp_max - disp_min)

    def q(v, M):
        return np.rint(np.fmin(np.fmax(v, f32(0)), f32(1)) * f32(M)).astype(np.uint32)

    def rgba(r, g, b):
        return (r | (g << 8) | (b << 16) | np.uint32(0xFF000000)).astype(np.uint32)

    if style == 0:
        g = q(t, 255)
        out = np.full(c.shape, 0xFF0000FF, np.uint32)  # unknown codes red
        ids = [0, 0xFFFF, 0xFFFE, 0xFFFC, 0xFFFD, 0xFFFB, 0xFFFA]
        for k, code in enumerate(ids):
            out[c == code] = colors[k]
        return np.where(disp, rgba(g, g, g), out).astype(np.uint32)
    if style == 2:
        with np.errstate(divide="ignore", invalid="ignore"):
            fb = f32(1) - np.fmin(t / f32(0.7), f32(1))
            fg = f32(1) - np.fmin(np.abs(t - f32(0.5)) / f32(0.59), f32(1))
            fr = f32(1) - np.fmin(np.abs(t - f32(0.8)) / f32(0.7), f32(1))
            fm = np.fmax(np.fmax(fr, fg), fb)
            col = rgba(q(fr / fm, 255), q(fg / fm, 255), q(fb / fm, 255))
        return np.where(disp, col, np.uint32(0xFF000000)).astype(np.uint32)
    if style == 1:
        return np.where(disp, q(t, 65535), 0).astype(np.uint16)
    if style == 3:
        return np.where(disp, c, 0).astype(np.uint16)
    return np.where(disp, (0x7FFF + inf_offset) - (c - 1), 0).astype(np.uint16)


def mipmap_layout(W, H):
    """Packed mip-map layout of a W x H map (DeviceSurfMipMap.h:78-120,
    DeviceSurfMipMap.cpp:68-146): -> (packed width, [(x, y, w, h) of level
    0 .. max]); the packed image is H rows high and max = len(rects) - 1."""
    nxt = lambda n: (n - 1) // 2 if n >= 1 else 0  # noqa: E731  C's (n - 1) / 2 for n >= 1
    x1 = (W // 4 + (1 if W % 4 else 0)) * 4
    rects, yy = [(0, 0, W, H)], 0
    w, h = W, H
    while nxt(w) > 0 and nxt(h) > 0:
        w, h = nxt(w), nxt(h)
        rects.append((x1, yy, w, h))
        yy += h
    return x1 + nxt(W), rects


def disp_mipmaps(codes, level_count=0, init=None):
    """Packed disparity mip-map (CreateDispMipMaps.cu:66-330 on the surface
    layout of DeviceSurfMipMap.h:78-120 / DeviceSurfMipMap.cpp:68-146) of a
    U16 EDisparityId code map, in float32 with the reference's operation
    order: CopyDispChannel (:90-114), then per level SmoothHorizontalLum
    (:117-176) into a temporary of width (W - 1) / 2 and SmoothVerticalLum
    (:179-238) with the 0.5 factor. `init` is the packed image before the
    call (pixels not written keep it; zeros if None). Returns (packed image,
    [(x, y, w, h) per level 0 .. max])."""
    f32 = np.float32
    c = np.asarray(codes).astype(np.int64)
    H, W = c.shape
    pw, rects = mipmap_layout(W, H)
    dims = [(w, h) for (_, _, w, h) in rects]
    max_levels = len(rects) - 1
    out = np.zeros((H, pw), f32) if init is None else np.array(init, f32, copy=True)
    if level_count > max_levels:
        raise ValueError("level count larger than the maximal possible level")
    if level_count <= 0:
        level_count = max_levels
    elif level_count == 1:
        return out, rects

    def mean121(a, b, cc):
        cnt = np.zeros(a.shape, f32)
        s = np.zeros(a.shape, f32)
        m = a != 0
        cnt = np.where(m, cnt + f32(1), cnt)
        s = np.where(m, s + a, s)
        m = b != 0
        cnt = np.where(m, cnt + f32(2), cnt)
        s = np.where(m, s + b * f32(2), s)
        m = cc != 0
        cnt = np.where(m, cnt + f32(1), cnt)
        s = np.where(m, s + cc, s)
        with np.errstate(divide="ignore", invalid="ignore"):
            return np.where(cnt > 0, s / cnt, f32(0)).astype(f32)

    lvl = np.where((c >= 1) & (c <= 0xFFEF), c, 0).astype(f32)
    out[:H, :W] = lvl
    for k in range(level_count - 1):
        w1, h1 = dims[k + 1]
        h0 = lvl.shape[0]
        tmp = mean121(lvl[:h0, 0:2 * w1:2], lvl[:h0, 1:2 * w1 + 1:2], lvl[:h0, 2:2 * w1 + 2:2])
        lvl = (f32(0.5) * mean121(tmp[0:2 * h1:2], tmp[1:2 * h1 + 1:2], tmp[2:2 * h1 + 2:2])).astype(f32)
        x, y, _, _ = rects[k + 1]
        out[y:y + h1, x:x + w1] = lvl
    return out, rects


def map3d(codes, cams, disp_min=1, disp_max=0xFFEF, cs_rut=False):
    """Disparity map -> 3D points (MapDisparityTo3D.cu:75-240) in float64 with
    explicit pinhole cameras, the library's replacement for the reference's
    _CStereoPinhole (not in the reference tree: parity of the camera model is
    unpinned). cams = [(fx, fy, cx, cy, R 3x3, centre 3)] * 2; codes are U16
    EDisparityId codes (float codes allowed for sub-pixel maps). Invalid codes
    use disparity disp_min, as the reference (:111-121). The rays through
    (x, y) and (x - d, y) meet at the midpoint of their closest points.
    Returns (H x W x 4 array (x, y, z, valid), (min xyz, max xyz) over the
    valid intersected points or None, mask of the pixels whose rays meet)."""
    c = np.asarray(codes, np.float64)
    H, W = c.shape
    valid = (c >= disp_min) & (c <= disp_max)
    d = np.where(valid, c - 1, float(disp_min))
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float64)

    def ray(cam, x, y):
        fx, fy, cx, cy, R, _ = cam
        v = np.stack([(x - cx) / fx, (y - cy) / fy, np.ones_like(x)], -1)
        return v @ np.asarray(R, np.float64).T

    dl, dr = ray(cams[0], xx, yy), ray(cams[1], xx - d, yy)
    oL, oR = np.asarray(cams[0][5], np.float64), np.asarray(cams[1][5], np.float64)
    n = np.cross(dl, dr)
    nn = (n * n).sum(-1)
    hit = nn > 1e-14 * (dl * dl).sum(-1) * (dr * dr).sum(-1)
    b = oR - oL
    with np.errstate(divide="ignore", invalid="ignore"):
        s = (np.cross(b, dr) * n).sum(-1) / nn
        t = (np.cross(b, dl) * n).sum(-1) / nn
    P = 0.5 * ((oL + s[..., None] * dl) + (oR + t[..., None] * dr))
    if cs_rut:
        P = P * np.array([1.0, -1.0, -1.0])
    out = np.zeros((H, W, 4))
    out[..., :3] = np.where(hit[..., None], P, 0.0)
    out[..., 3] = np.where(hit & valid, 1.0, 0.0)
    good = hit & valid
    rng = (P[good].min(0), P[good].max(0)) if good.any() else None
    return out, rng, hit


def crosscheck(base, other, tol=1, left_to_right=True):
    """-> (out int16 with -2 = inconsistent, (min, max))"""
    base = np.ascontiguousarray(base, np.int16)
    other = np.ascontiguousarray(other, np.int16)
    H, W = base.shape
    out = np.empty((H, W), np.int16)
    rng = np.zeros(2, np.int32)
    lib().or_crosscheck(_p(base), _p(other), W, H, tol, 1 if left_to_right else 0, _p(out), _p(rng))
    return out, (int(rng[0]), int(rng[1]))


def div_int_mismatches(d, nmax=1 << 24):
    """Integers |x| <= nmax for which the reference-compat kernel's
    constant-divisor quotient (multiply by RN(1/d), one remainder correction)
    differs from the IEEE binary32 quotient x / d."""
    return int(lib().or_div_int_mismatches(d, nmax))


def box_sums(data, kx, ky):
    """int32 box sums of every kx x ky window inside `data`, anchored at the
    window's top-left pixel (the matchers' aggregation): (H-ky+1, W-kx+1)."""
    d = np.ascontiguousarray(data, np.int32)
    H, W = d.shape
    out = np.zeros((H - ky + 1, W - kx + 1), np.int32)
    lib().or_box_sums(_p(d), W, H, kx, ky, _p(out))
    return out


def crosscheck_codes(base, other, tol=1, left_to_right=True, frame=True, out=None):
    """The reference's rule on uint16 EDisparityId codes (raw code compare).
    frame=True leaves the 1-pixel frame of `out` as given (zeros if out is
    None). -> (out uint16, (min code, max code)); (0xFFEF, 1) when none kept."""
    base = np.ascontiguousarray(base, np.uint16)
    other = np.ascontiguousarray(other, np.uint16)
    H, W = base.shape
    res = np.zeros((H, W), np.uint16) if out is None else np.array(out, np.uint16, copy=True)
    rng = np.zeros(2, np.int32)
    lib().or_crosscheck_codes(_p(base), _p(other), W, H, tol, 1 if left_to_right else 0, 1 if frame else 0,
                              _p(res), _p(rng))
    return res, (int(rng[0]), int(rng[1]))


# ---- encodings of the library's output maps --------------------------------

def to_u8(disp):
    """int16 oracle map -> the library's U8 encoding (255 = not a disparity)."""
    d = np.asarray(disp)
    return np.where(d >= 0, d, 255).astype(np.uint8)


def to_u16(disp):
    """int16 oracle map -> EDisparityId U16 encoding (d+1; 0xFFFF cannot
    evaluate; 0xFFFA inconsistent)."""
    d = np.asarray(disp).astype(np.int32)
    out = np.where(d >= 0, d + 1, 0xFFFF)
    out = np.where(d == -2, 0xFFFA, out)
    return out.astype(np.uint16)


COMPAT_METHODS = {"sad1": 0, "ncc": 1, "aw1": 2, "aw2": 3, "bm1": 4}


def compat_match(L, R, method, D, patch, dmin=0, sim_type=0, left_to_right=True, grad_thresh=0.0,
                 score_thresh=0.0, min_delta_thresh=0.0):
    """The reference matchers' 4 x uint16 output (oracle/compat.cpp):
    method in COMPAT_METHODS; patch = window side (SAD1, NCC, BM1) or
    sub-window side (AW1, AW2). -> (H, W, 4) uint16: x = disparity + 1 or an
    EDisparityId, y = score, z / w = specificity."""
    L, R = _u8(L), _u8(R)
    H, W = L.shape
    out = np.empty((H, W, 4), np.uint16)
    lib().or_compat_match(_p(L), _p(R), W, H, W, COMPAT_METHODS[method], D, dmin, patch, sim_type,
                          1 if left_to_right else 0, grad_thresh, score_thresh, min_delta_thresh, _p(out))
    return out


def gate_mask(img, kind, P, thresh):
    """Gradient gate of the plain matchers (oracle/compat.cpp or_gate_mask):
    kind 0 mean |dI/dx| (SAD1, NCC), 1 standard deviation in % (AW1) over
    the P x P patch -> bool (H, W), True where the pixel is gated."""
    img = _u8(img)
    H, W = img.shape
    m = np.empty((H, W), np.uint8)
    lib().or_gate_mask(_p(img), W, H, W, kind, P, thresh, _p(m))
    return m.astype(bool)
