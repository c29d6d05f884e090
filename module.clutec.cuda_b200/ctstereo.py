"""ctstereo — Python mirror of the CluTec.Cuda MultiView driver API over the
libctstereo C ABI (include/ctstereo.h).

Each reference driver (``BlockMatcherNCC::CDriver`` etc.) is a class with
``configure(device, fmt, params)`` and ``process(...)``; images are torch CUDA
tensors (uint8 / int16-as-uint16 / int64-as-uint64 / float32, 2-D, row-major,
rows 16-byte aligned). Errors raise :class:`CtError`, the counterpart of the
reference's ``CLU_EXCEPTION``. All calls are asynchronous on the given CUDA
stream (default: torch's current stream).

The native library must be built (``python module.clutec.cuda_b200/build.py``);
there is no fallback path: loading fails loudly if the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libctstereo.so"
SYNTH_PATH = _PKG / "libctsynth.so"

# status codes (ctstereo.h)
CT_OK, CT_EINVAL, CT_ETYPE, CT_EFORMAT, CT_ECUDA, CT_ETIMEOUT, CT_ESTATE, CT_ENOMEM, CT_EINTERNAL = range(9)
# pixel types
CT_PIX_U8, CT_PIX_U16, CT_PIX_U64, CT_PIX_F32, CT_PIX_RGBA8, CT_PIX_F32X4, CT_PIX_U16X4 = 1, 2, 3, 4, 5, 6, 7
CT_COMPAT_SAD1, CT_COMPAT_NCC, CT_COMPAT_AW1, CT_COMPAT_AW2, CT_COMPAT_BM1 = 0, 1, 2, 3, 4
CT_COLOR_ANALYSIS, CT_COLOR_GRAY, CT_COLOR_COLOR, CT_COLOR_DISP_ABS, CT_COLOR_DISP_REL = range(5)
# EDisparityId codes
DISP_FIRST, DISP_LAST = 0x0001, 0xFFEF
DISP_CANNOT_EVALUATE, DISP_INCONSISTENT, DISP_U8_INVALID = 0xFFFF, 0xFFFA, 0xFF
CENSUS_9X7, CENSUS_3X3 = 0, 1

_STATUS_NAMES = {0: "CT_OK", 1: "CT_EINVAL", 2: "CT_ETYPE", 3: "CT_EFORMAT", 4: "CT_ECUDA",
                 5: "CT_ETIMEOUT", 6: "CT_ESTATE", 7: "CT_ENOMEM", 8: "CT_EINTERNAL"}


class CtError(RuntimeError):
    """A non-zero status from the C ABI, with ct_last_error_string()."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{_STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class ct_image(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("pitch_bytes", C.c_size_t), ("width", C.c_int32),
                ("height", C.c_int32), ("type", C.c_int32), ("reserved", C.c_int32)]


class ct_format(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("type", C.c_int32)]


class ct_census_params(C.Structure):
    _fields_ = [("window", C.c_int32)]


class ct_census_match_params(C.Structure):
    _fields_ = [("disp_count", C.c_int32), ("agg_radius", C.c_int32), ("left_to_right", C.c_int32),
                ("disp_min", C.c_int32)]


class ct_sad_params(C.Structure):
    _fields_ = [("disp_count", C.c_int32), ("radius", C.c_int32), ("left_to_right", C.c_int32),
                ("disp_min", C.c_int32)]


class ct_ncc_params(C.Structure):
    _fields_ = [("disp_count", C.c_int32), ("radius", C.c_int32), ("left_to_right", C.c_int32),
                ("disp_min", C.c_int32)]


class ct_aw_params(C.Structure):
    _fields_ = [("disp_count", C.c_int32), ("left_to_right", C.c_int32), ("disp_min", C.c_int32),
                ("reserved1", C.c_int32)]


class ct_compat_params(C.Structure):
    _fields_ = [("method", C.c_int32), ("disp_count", C.c_int32), ("disp_min", C.c_int32), ("patch", C.c_int32),
                ("sim_type", C.c_int32), ("left_to_right", C.c_int32), ("grad_thresh", C.c_float),
                ("score_thresh", C.c_float), ("min_delta_thresh", C.c_float), ("reserved", C.c_int32 * 3)]


class ct_pinhole(C.Structure):
    _fields_ = [("fx", C.c_float), ("fy", C.c_float), ("cx", C.c_float), ("cy", C.c_float),
                ("rot", C.c_float * 9), ("center", C.c_float * 3)]


class ct_map3d_params(C.Structure):
    _fields_ = [("disp_min", C.c_int32), ("disp_max", C.c_int32), ("cs_rut", C.c_int32), ("reserved", C.c_int32),
                ("cam", ct_pinhole * 2)]


class ct_crosscheck_params(C.Structure):
    _fields_ = [("disp_delta_thresh", C.c_int32), ("left_to_right", C.c_int32), ("reserved0", C.c_int32),
                ("reserved1", C.c_int32)]


class ct_batch_shape(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("disp_count", C.c_int32), ("reserved", C.c_int32)]


class ct_batch_item(C.Structure):
    _fields_ = [("left", ct_image), ("right", ct_image), ("disp", ct_image)]


class ct_curves(C.Structure):
    _fields_ = [("ptr", C.c_void_p), ("pitch_bytes", C.c_size_t), ("width", C.c_int32), ("height", C.c_int32),
                ("disp_count", C.c_int32), ("reserved", C.c_int32)]


class ct_color_params(C.Structure):
    _fields_ = [("style", C.c_int32), ("disp_min", C.c_int32), ("disp_max", C.c_int32), ("inf_offset", C.c_int32),
                ("colors", C.c_uint32 * 7)]


CT_CONFNET_PARAMS = 12673


class ct_pipe_rates(C.Structure):
    _fields_ = [("popc_per_clk_sm", C.c_double), ("iadd3_per_clk_sm", C.c_double),
                ("lop3_per_clk_sm", C.c_double), ("vimnmx_per_clk_sm", C.c_double),
                ("imad_per_clk_sm", C.c_double), ("sm_clock_mhz", C.c_double), ("sm_count", C.c_int32),
                ("reserved", C.c_int32)]


_lib = None


def lib() -> C.CDLL:
    """Loads libctstereo.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} not built: run python module.clutec.cuda_b200/build.py")
        _lib = C.CDLL(str(LIB_PATH))
        _declare(_lib)
    return _lib


def _declare(L: C.CDLL) -> None:
    H = C.c_void_p
    P = C.POINTER
    img = P(ct_image)
    fmt = P(ct_format)
    L.ct_last_error_string.restype = C.c_char_p
    L.ct_version.restype = C.c_char_p
    sigs = {
        "ct_destroy": [H],
        "ct_handle_device_status": [H, P(C.c_int32)],
        "ct_census_create": [P(H)],
        "ct_census_configure": [H, C.c_int32, fmt, P(ct_census_params)],
        "ct_census_process": [H, img, img, C.c_void_p],
        "ct_census_process_pair": [H, img, img, img, img, C.c_void_p],
        "ct_bm_census_create": [P(H)],
        "ct_bm_census_configure": [H, C.c_int32, fmt, P(ct_census_match_params)],
        "ct_bm_census_process": [H, img, img, img, C.c_void_p],
        "ct_bm_census_process_lr": [H, img, img, img, C.c_int32, img, img, C.c_void_p],
        "ct_bm_census_match_desc": [H, img, img, img, C.c_int32, C.c_void_p],
        "ct_bm_census_autotune": [H, img, img, C.c_void_p],
        "ct_bm_census_tuning": [H, P(C.c_int32), P(C.c_int32)],
        "ct_bm_census_set_tuning": [H, C.c_int32, C.c_int32],
        "ct_bm_census_set_fused_lr": [H, C.c_int32],
        "ct_bm_ncc_set_tensor_cores": [H, C.c_int32],
        "ct_bm_census_process_static": [img, img, img, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p],
        "ct_bm_census_static_status": [P(C.c_int32)],
        "ct_bm_set_gradient_gate": [H, C.c_float],
        "ct_bm_compat_create": [P(H)],
        "ct_bm_compat_configure": [H, C.c_int32, fmt, P(ct_compat_params)],
        "ct_bm_compat_process": [H, img, img, img, C.c_void_p],
        "ct_handle_test_wait_timeout": [H, C.c_uint32, C.c_void_p],
        "ct_curves_pitch": [C.c_int32, P(C.c_size_t)],
        "ct_bm_census_process_curves": [H, img, P(ct_curves), img, img, C.c_void_p],
        "ct_confnet_create": [P(H)],
        "ct_confnet_configure": [H, C.c_int32, C.c_int32],
        "ct_confnet_init": [H, C.c_uint64],
        "ct_confnet_set_params": [H, C.c_void_p, C.c_int32],
        "ct_confnet_get_params": [H, C.c_void_p, C.c_int32],
        "ct_confnet_gather": [H, C.c_void_p, P(ct_curves), img, C.c_void_p, C.c_int32, C.c_void_p],
        "ct_confnet_loss_grad": [H, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p],
        "ct_confnet_train_step": [H, C.c_void_p, C.c_void_p, C.c_int32, C.c_float, C.c_void_p, C.c_void_p],
        "ct_confnet_scores": [H, C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p],
        "ct_confnet_infer": [H, img, P(ct_curves), img, img, C.c_float, C.c_void_p],
        "ct_bm_sad_create": [P(H)],
        "ct_bm_sad_configure": [H, C.c_int32, fmt, P(ct_sad_params)],
        "ct_bm_sad_process": [H, img, img, img, C.c_void_p],
        "ct_bm_ncc_create": [P(H)],
        "ct_bm_ncc_configure": [H, C.c_int32, fmt, P(ct_ncc_params)],
        "ct_bm_ncc_process": [H, img, img, img, img, img, C.c_void_p],
        "ct_bm_aw_create": [P(H)],
        "ct_bm_aw_configure": [H, C.c_int32, fmt, P(ct_aw_params)],
        "ct_bm_aw_process": [H, img, img, img, C.c_void_p],
        "ct_bm_aw_process_guided": [H, img, img, img, img, C.c_void_p],
        "ct_crosscheck_create": [P(H)],
        "ct_crosscheck_configure": [H, C.c_int32, fmt, P(ct_crosscheck_params)],
        "ct_crosscheck_process": [H, img, img, img, C.c_void_p],
        "ct_crosscheck_range": [H, P(C.c_int32), P(C.c_int32)],
        "ct_map3d_create": [P(H)],
        "ct_map3d_configure": [H, C.c_int32, fmt, P(ct_map3d_params)],
        "ct_map3d_process": [H, img, img, C.c_void_p],
        "ct_map3d_range": [H, P(C.c_float), P(C.c_float)],
        "ct_batch_create": [P(H)],
        "ct_batch_configure": [H, C.c_int32, P(ct_batch_shape), C.c_int32, C.c_int32],
        "ct_batch_process": [H, P(ct_batch_item), C.c_int32, C.c_void_p],
        "ct_batch_autotune": [H, P(ct_batch_item), C.c_int32, C.c_void_p],
        "ct_batch_strip_height": [H, C.c_int32, P(C.c_int32)],
        "ct_batch_graph_create": [H, P(ct_batch_item), C.c_int32],
        "ct_batch_graph_launch": [H, C.c_void_p],
        "ct_color_params_default": [C.c_int32, P(ct_color_params)],
        "ct_color_disparity": [img, img, P(ct_color_params), C.c_void_p],
        "ct_disp_mipmap_format": [C.c_int32, C.c_int32, P(C.c_int32), P(C.c_int32)],
        "ct_disp_mipmap_level": [C.c_int32, C.c_int32, C.c_int32, P(C.c_int32), P(C.c_int32), P(C.c_int32),
                                 P(C.c_int32)],
        "ct_disp_mipmaps": [img, img, C.c_int32, C.c_void_p],
        "ct_census_stream_create": [P(H)],
        "ct_census_stream_configure": [H, C.c_int32, fmt, P(ct_census_match_params), C.c_int32, C.c_int32],
        "ct_census_stream_submit": [H, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                                    P(C.c_int64)],
        "ct_census_stream_wait": [H, C.c_int64],
        "ct_census_stream_timer_start": [H],
        "ct_census_stream_timer_stop": [H, P(C.c_float)],
        "ct_probe_pipe_rates": [C.c_int32, P(ct_pipe_rates)],
    }
    for name, args in sigs.items():
        f = getattr(L, name, None)
        if f is None:
            continue
        f.argtypes = args
        f.restype = C.c_int


def exported_symbols(header: str = "ctstereo.h"):
    """Names of the ct_* entry points declared in include/<header>."""
    hdr = (_PKG.parent / "include" / header).read_text()
    return sorted(set(re.findall(r"^(?:int|const char\s*\*)\s+(ct_[a-z0-9_]+)\s*\(", hdr, re.M)))


def check(rc: int) -> None:
    if rc != CT_OK:
        raise CtError(rc, lib().ct_last_error_string().decode())


def version() -> str:
    return lib().ct_version().decode()


# ---------------------------------------------------------------------------
# tensors <-> ct_image
# ---------------------------------------------------------------------------

def _pix_type(t) -> int:
    import torch
    m = {torch.uint8: CT_PIX_U8, torch.int16: CT_PIX_U16, torch.uint16: CT_PIX_U16,
         torch.int64: CT_PIX_U64, torch.uint64: CT_PIX_U64, torch.float32: CT_PIX_F32}
    if t.dtype not in m:
        raise CtError(CT_ETYPE, f"tensor dtype {t.dtype} has no ctstereo pixel type")
    return m[t.dtype]


def image(t, type_=None) -> ct_image:
    """Describes a 2-D CUDA tensor (row stride may exceed the width) as a
    ct_image; type_ overrides the pixel type (CT_PIX_RGBA8 for an int32 or
    uint32 tensor of packed r, g, b, a bytes)."""
    if t.dim() != 2 or t.stride(1) != 1:
        raise CtError(CT_EINVAL, "images must be 2-D tensors with unit column stride")
    return ct_image(t.data_ptr(), t.stride(0) * t.element_size(), t.shape[1], t.shape[0],
                    _pix_type(t) if type_ is None else type_, 0)


def _img_ref(t):
    return None if t is None else C.byref(image(t))


def _stream(stream):
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


def alloc_image(height: int, width: int, dtype, device="cuda"):
    """A 2-D tensor whose row pitch is a multiple of 256 bytes (TMA-friendly)."""
    import torch
    esz = torch.empty(0, dtype=dtype).element_size()
    pitch = -(-width * esz // 256) * 256 // esz
    return torch.empty((height, pitch), dtype=dtype, device=device)[:, :width]


class _Driver:
    _create = None

    def __init__(self):
        h = C.c_void_p()
        check(getattr(lib(), self._create)(C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().ct_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def device_status(self) -> int:
        v = C.c_int32()
        check(lib().ct_handle_device_status(self._h, C.byref(v)))
        return v.value

    def set_gradient_gate(self, grad_thresh: float):
        """ct_bm_set_gradient_gate (SAD, NCC and AW matchers): pixels whose
        patch has too little texture get no disparity."""
        check(lib().ct_bm_set_gradient_gate(self._h, grad_thresh))

    def test_wait_timeout(self, poll_limit: int = 1024, stream=None):
        """ct_handle_test_wait_timeout: a bounded device wait that nothing
        completes gives up and sets this handle's status to CT_ETIMEOUT."""
        check(lib().ct_handle_test_wait_timeout(self._h, poll_limit, _stream(stream)))


def _fmt(width, height, type_=CT_PIX_U8):
    return ct_format(width, height, type_)


class CensusTransform(_Driver):
    """CensusTransform::CDriver (CensusTransform.h:44-70)."""
    _create = "ct_census_create"

    def configure(self, device: int, width: int, height: int, window: int = CENSUS_9X7):
        check(lib().ct_census_configure(self._h, device, C.byref(_fmt(width, height)),
                                        C.byref(ct_census_params(window))))

    def process(self, dst, src, stream=None):
        check(lib().ct_census_process(self._h, _img_ref(dst), _img_ref(src), _stream(stream)))

    def process_pair(self, dst_left, dst_right, src_left, src_right, stream=None):
        """Both views in one launch (9x7 only)."""
        check(lib().ct_census_process_pair(self._h, _img_ref(dst_left), _img_ref(dst_right), _img_ref(src_left),
                                           _img_ref(src_right), _stream(stream)))


class BlockMatcherCensus(_Driver):
    """Census (9x7 / 64-bit) + Hamming + 5x5 box + WTA matcher."""
    _create = "ct_bm_census_create"

    def configure(self, device: int, width: int, height: int, disp_count: int, left_to_right: bool = True,
                  agg_radius: int = 2, disp_min: int = 0):
        """Disparities disp_min .. disp_min + disp_count - 1."""
        check(lib().ct_bm_census_configure(self._h, device, C.byref(_fmt(width, height)), C.byref(
            ct_census_match_params(disp_count, agg_radius, int(left_to_right), disp_min))))

    def process(self, disp, left, right, stream=None):
        check(lib().ct_bm_census_process(self._h, _img_ref(disp), _img_ref(left), _img_ref(right),
                                         _stream(stream)))

    def autotune(self, left, right, stream=None):
        """Times the launch-shape candidates on these images; keeps the fastest."""
        check(lib().ct_bm_census_autotune(self._h, _img_ref(left), _img_ref(right), _stream(stream)))
        return self.tuning()

    def set_tuning(self, strip_height: int, disp_per_warp: int):
        check(lib().ct_bm_census_set_tuning(self._h, strip_height, disp_per_warp))

    def set_fused_lr(self, enable: bool):
        """process_lr in one matching pass (default) or two (one per direction); same maps."""
        check(lib().ct_bm_census_set_fused_lr(self._h, 1 if enable else 0))

    def tuning(self):
        th, dpw = C.c_int32(), C.c_int32()
        check(lib().ct_bm_census_tuning(self._h, C.byref(th), C.byref(dpw)))
        return {"strip_height": th.value, "disp_per_warp": dpw.value}

    def match_desc(self, disp, desc_base, desc_match, left_to_right=True, stream=None):
        """Matching on precomputed 9x7 census descriptors (int64 tensors)."""
        check(lib().ct_bm_census_match_desc(self._h, _img_ref(disp), _img_ref(desc_base), _img_ref(desc_match),
                                            int(left_to_right), _stream(stream)))

    def process_lr(self, left, right, disp_lr=None, disp_rl=None, disp_checked=None, tol=1, stream=None):
        check(lib().ct_bm_census_process_lr(self._h, _img_ref(disp_lr), _img_ref(disp_rl),
                                            _img_ref(disp_checked), tol, _img_ref(left), _img_ref(right),
                                            _stream(stream)))

    def process_curves(self, disp, curves, left, right, stream=None):
        """process() that also writes the cost-curve volume (see CurveVolume)."""
        check(lib().ct_bm_census_process_curves(self._h, _img_ref(disp), C.byref(curves.desc()), _img_ref(left),
                                                _img_ref(right), _stream(stream)))


class CurveVolume:
    """Device cost-curve volume (ct_curves): rows (y, g) of 32-bit words, word
    x + 2 of row (y, g) = codes of disparities 4g .. 4g + 3 at column x."""

    def __init__(self, width: int, height: int, disp_count: int, device="cuda"):
        import torch
        pitch = C.c_size_t()
        check(lib().ct_curves_pitch(width, C.byref(pitch)))
        self.width, self.height, self.disp_count = width, height, disp_count
        self.groups = (disp_count + 3) // 4
        self.pitch_words = pitch.value // 4
        self.words = torch.full((height * self.groups, self.pitch_words), -1, dtype=torch.int32, device=device)

    def desc(self) -> ct_curves:
        return ct_curves(self.words.data_ptr(), self.pitch_words * 4, self.width, self.height, self.disp_count, 0)

    def to_hwd(self):
        """(H, W, D) uint8 numpy array of the codes."""
        import numpy as np
        w = self.words.cpu().numpy().view(np.uint32).reshape(self.height, self.groups, self.pitch_words)
        b = w[:, :, 2:2 + self.width].view(np.uint8).reshape(self.height, self.groups, self.width, 4)
        return np.ascontiguousarray(b.transpose(0, 2, 1, 3).reshape(self.height, self.width, 4 * self.groups)
                                    [:, :, :self.disp_count])


class BlockMatcherSAD1(_Driver):
    """BlockMatcherSAD1::CDriver, exhaustive (2r+1)^2 SAD + WTA."""
    _create = "ct_bm_sad_create"

    def configure(self, device: int, width: int, height: int, disp_count: int, radius: int = 4,
                  left_to_right: bool = True, disp_min: int = 0):
        check(lib().ct_bm_sad_configure(self._h, device, C.byref(_fmt(width, height)),
                                        C.byref(ct_sad_params(disp_count, radius, int(left_to_right), disp_min))))

    def process(self, disp, left, right, stream=None):
        check(lib().ct_bm_sad_process(self._h, _img_ref(disp), _img_ref(left), _img_ref(right),
                                      _stream(stream)))


class BlockMatcherNCC(_Driver):
    """BlockMatcherNCC::CDriver with an FP32 (unquantised) score."""
    _create = "ct_bm_ncc_create"

    def configure(self, device: int, width: int, height: int, disp_count: int, radius: int = 5,
                  disp_min: int = 0):
        check(lib().ct_bm_ncc_configure(self._h, device, C.byref(_fmt(width, height)),
                                        C.byref(ct_ncc_params(disp_count, radius, 1, disp_min))))

    def process(self, disp, left, right, score=None, disp_init=None, stream=None):
        check(lib().ct_bm_ncc_process(self._h, _img_ref(disp), _img_ref(score), _img_ref(left),
                                      _img_ref(right), _img_ref(disp_init), _stream(stream)))

    def set_tensor_cores(self, enable: bool):
        """Unguided matching on the tensor cores (default) or on the CUDA cores; same maps."""
        check(lib().ct_bm_ncc_set_tensor_cores(self._h, 1 if enable else 0))


class BlockMatcherAW(_Driver):
    """BlockMatcherAW1/AW2: best of 5 shifted 7x7 SAD windows + sub-pixel."""
    _create = "ct_bm_aw_create"

    def configure(self, device: int, width: int, height: int, disp_count: int, disp_min: int = 0):
        check(lib().ct_bm_aw_configure(self._h, device, C.byref(_fmt(width, height)),
                                       C.byref(ct_aw_params(disp_count, 1, disp_min, 0))))

    def process(self, disp, left, right, disp_init=None, stream=None):
        """disp_init: coarse disparity map of the guided mode (or None)."""
        if disp_init is None:
            check(lib().ct_bm_aw_process(self._h, _img_ref(disp), _img_ref(left), _img_ref(right),
                                         _stream(stream)))
        else:
            check(lib().ct_bm_aw_process_guided(self._h, _img_ref(disp), _img_ref(left), _img_ref(right),
                                                _img_ref(disp_init), _stream(stream)))


class CrossCheckDisparityMaps(_Driver):
    """CrossCheckDisparityMaps::CDriver."""
    _create = "ct_crosscheck_create"

    def configure(self, device: int, width: int, height: int, type_: int = CT_PIX_U8,
                  disp_delta_thresh: int = 1, left_to_right: bool = True):
        check(lib().ct_crosscheck_configure(self._h, device, C.byref(_fmt(width, height, type_)),
                                            C.byref(ct_crosscheck_params(disp_delta_thresh,
                                                                         int(left_to_right), 0, 0))))

    def process(self, result, disp_base, disp_other, stream=None):
        check(lib().ct_crosscheck_process(self._h, _img_ref(result), _img_ref(disp_base),
                                          _img_ref(disp_other), _stream(stream)))

    def disp_range(self):
        lo, hi = C.c_int32(), C.c_int32()
        check(lib().ct_crosscheck_range(self._h, C.byref(lo), C.byref(hi)))
        return lo.value, hi.value


def pinhole(fx, fy, cx, cy, rot=None, center=(0.0, 0.0, 0.0)) -> ct_pinhole:
    """A pinhole camera: focal lengths and principal point in pixels,
    camera-to-world rotation (3x3, row-major; identity if None) and the
    projection centre in world coordinates."""
    r = [1, 0, 0, 0, 1, 0, 0, 0, 1] if rot is None else [float(v) for row in rot for v in row]
    return ct_pinhole(fx, fy, cx, cy, (C.c_float * 9)(*r), (C.c_float * 3)(*center))


def alloc_u16x4(height: int, width: int, device="cuda"):
    """A (height, width, 4) int16 tensor with a 256-byte aligned row pitch for
    the reference matchers' 4 x uint16 pixels (BlockMatcherCompat)."""
    import torch
    return alloc_image(height, 4 * width, torch.int16, device).unflatten(1, (width, 4))


def _u16x4_ref(t):
    """ct_image of a (H, W, 4) int16 tensor (CT_PIX_U16X4), or of a 2-D U16 map."""
    if t.dim() == 2:
        return C.byref(image(t))
    if t.dim() != 3 or t.shape[2] != 4 or t.stride(2) != 1 or t.stride(1) != 4 or t.element_size() != 2:
        raise CtError(CT_EINVAL, "4 x uint16 images must be (H, W, 4) 16-bit tensors with packed pixels")
    return C.byref(ct_image(t.data_ptr(), t.stride(0) * 2, t.shape[1], t.shape[0], CT_PIX_U16X4, 0))


class BlockMatcherCompat(_Driver):
    """The reference matchers' own 4 x uint16 output (ct_bm_compat_*):
    method CT_COMPAT_SAD1 / NCC / AW1 / AW2 / BM1 with their gates, thresholds
    and scan bookkeeping; patch = window side (SAD1, NCC, BM1) or sub-window
    side (AW1, AW2)."""
    _create = "ct_bm_compat_create"

    def configure(self, device: int, width: int, height: int, method: int, disp_count: int, patch: int,
                  disp_min: int = 0, sim_type: int = 0, left_to_right: bool = True, grad_thresh: float = 0.0,
                  score_thresh: float = 0.0, min_delta_thresh: float = 0.0):
        p = ct_compat_params(method, disp_count, disp_min, patch, sim_type, int(left_to_right), grad_thresh,
                             score_thresh, min_delta_thresh)
        check(lib().ct_bm_compat_configure(self._h, device, C.byref(_fmt(width, height)), C.byref(p)))

    def process(self, disp, left, right, stream=None):
        """disp: alloc_u16x4 tensor (all channels) or a 2-D int16 map (x only)."""
        check(lib().ct_bm_compat_process(self._h, _u16x4_ref(disp), _img_ref(left), _img_ref(right),
                                         _stream(stream)))


def alloc_map3d(height: int, width: int, device="cuda"):
    """A (height, width, 4) float32 tensor with a 256-byte aligned row pitch
    (x, y, z, valid per pixel)."""
    import torch
    return alloc_image(height, 4 * width, torch.float32, device).unflatten(1, (width, 4))


class MapDisparityTo3D(_Driver):
    """MapDisparityTo3D::CDriver with explicit pinhole cameras (ct_map3d_*)."""
    _create = "ct_map3d_create"

    def configure(self, device: int, width: int, height: int, cam_left: ct_pinhole, cam_right: ct_pinhole,
                  disp_min: int = 1, disp_max: int = 0xFFEF, cs_rut: bool = False, type_: int = CT_PIX_U16):
        p = ct_map3d_params(disp_min, disp_max, int(cs_rut), 0, (ct_pinhole * 2)(cam_left, cam_right))
        check(lib().ct_map3d_configure(self._h, device, C.byref(_fmt(width, height, type_)), C.byref(p)))

    def process(self, map3d, disp, stream=None):
        """map3d: a (H, W, 4) float32 CUDA tensor (alloc_map3d)."""
        if map3d.dim() != 3 or map3d.shape[2] != 4 or map3d.stride(2) != 1 or map3d.stride(1) != 4:
            raise CtError(CT_EINVAL, "map3d must be (H, W, 4) float32 with packed pixels")
        m = ct_image(map3d.data_ptr(), map3d.stride(0) * 4, map3d.shape[1], map3d.shape[0], CT_PIX_F32X4, 0)
        check(lib().ct_map3d_process(self._h, C.byref(m), _img_ref(disp), _stream(stream)))

    def range(self):
        """(min xyz, max xyz) of the valid points of the last call (synchronises)."""
        lo, hi = (C.c_float * 3)(), (C.c_float * 3)()
        check(lib().ct_map3d_range(self._h, lo, hi))
        return tuple(lo), tuple(hi)


class BatchStereo(_Driver):
    """Batched census stereo (both directions + cross-check) over many pairs:
    one census launch and one persistent matching launch per call."""
    _create = "ct_batch_create"

    def configure(self, device: int, shapes, tol: int = 1):
        """shapes: list of (width, height, disp_count)."""
        arr = (ct_batch_shape * len(shapes))(*[ct_batch_shape(w, h, d, 0) for w, h, d in shapes])
        check(lib().ct_batch_configure(self._h, device, arr, len(shapes), tol))
        self.n = len(shapes)

    @staticmethod
    def _items(pairs):
        """pairs: list of (left, right, disp) tensors."""
        return (ct_batch_item * len(pairs))(*[ct_batch_item(image(l), image(r), image(d)) for l, r, d in pairs])

    def process(self, pairs, stream=None):
        items = self._items(pairs)
        check(lib().ct_batch_process(self._h, items, len(pairs), _stream(stream)))

    def autotune(self, pairs, stream=None):
        items = self._items(pairs)
        check(lib().ct_batch_autotune(self._h, items, len(pairs), _stream(stream)))
        return self.strip_heights()

    def strip_heights(self):
        out = []
        for i in range(self.n):
            v = C.c_int32()
            check(lib().ct_batch_strip_height(self._h, i, C.byref(v)))
            out.append(v.value)
        return out

    def graph_create(self, pairs):
        self._graph_items = self._items(pairs)  # keep the descriptors alive
        check(lib().ct_batch_graph_create(self._h, self._graph_items, len(pairs)))

    def graph_launch(self, stream=None):
        check(lib().ct_batch_graph_launch(self._h, _stream(stream)))


def color_params(style: int) -> ct_color_params:
    """ColorDisparityImage::SParameter defaults for a style."""
    p = ct_color_params()
    check(lib().ct_color_params_default(style, C.byref(p)))
    return p


def color_disparity(out, disp, params: ct_color_params, stream=None):
    """ColorDisparityImage::CDriver::Process: out is an int32 tensor (RGBA8
    styles, bytes r, g, b, a) or uint16/int16 (the U16 styles)."""
    rgba = params.style in (CT_COLOR_ANALYSIS, CT_COLOR_COLOR)
    o = image(out, CT_PIX_RGBA8 if rgba else None)
    check(lib().ct_color_disparity(C.byref(o), _img_ref(disp), C.byref(params), _stream(stream)))


def disp_mipmap_format(width: int, height: int):
    """-> (packed image width, maximal level count) of the packed mip-map of a
    width x height disparity map (CDeviceSurfMipMap::Create,
    DeviceSurfMipMap.cpp:68-146); the packed image is `height` rows high."""
    pw, n = C.c_int32(), C.c_int32()
    check(lib().ct_disp_mipmap_format(width, height, C.byref(pw), C.byref(n)))
    return pw.value, n.value


def disp_mipmap_level(width: int, height: int, level: int):
    """-> (x, y, w, h) of a level in the packed mip-map
    (_CDeviceSurfMipMap::GetOrigin / Format)."""
    v = [C.c_int32() for _ in range(4)]
    check(lib().ct_disp_mipmap_level(width, height, level, *[C.byref(x) for x in v]))
    return tuple(x.value for x in v)


def disp_mipmaps(mipmap, disp, level_count: int = 0, stream=None):
    """CreateDispMipMaps::CDriver::Run: mipmap is a float32 CUDA tensor of the
    packed size, disp a uint8 or int16/uint16 disparity map."""
    check(lib().ct_disp_mipmaps(C.byref(image(mipmap)), _img_ref(disp), level_count, _stream(stream)))


class CensusStream(_Driver):
    """Streamed census stereo (ct_census_stream_*): host frames in, host
    cross-checked maps out, copies of neighbouring frames overlapping the
    matching. Host images are 2-D CPU tensors (pin_memory() ones overlap)."""
    _create = "ct_census_stream_create"

    def configure(self, device: int, width: int, height: int, disp_count: int, tol: int = 1, out_type=None):
        import torch
        self.out_dtype = torch.uint8 if out_type in (None, torch.uint8) else torch.int16
        ot = CT_PIX_U8 if self.out_dtype == torch.uint8 else CT_PIX_U16
        check(lib().ct_census_stream_configure(self._h, device, C.byref(_fmt(width, height)),
                                               C.byref(ct_census_match_params(disp_count, 2, 1, 0)), tol, ot))
        self._held = {}

    @staticmethod
    def _host(t):
        if t.device.type != "cpu" or t.dim() != 2 or t.stride(1) != 1:
            raise CtError(CT_EINVAL, "host images must be 2-D CPU tensors with unit column stride")
        return C.c_void_p(t.data_ptr()), t.stride(0) * t.element_size()

    def submit(self, left, right, checked) -> int:
        """Enqueues a frame; returns its number. The tensors stay referenced
        (and must stay unchanged) until wait() for that frame."""
        (pl, sl), (pr, sr), (po, so) = self._host(left), self._host(right), self._host(checked)
        k = C.c_int64()
        check(lib().ct_census_stream_submit(self._h, pl, sl, pr, sr, po, so, C.byref(k)))
        self._held[k.value] = (left, right, checked)
        return k.value

    def wait(self, frame: int):
        check(lib().ct_census_stream_wait(self._h, frame))
        for f in [f for f in self._held if f <= frame]:
            del self._held[f]

    def timer_start(self):
        check(lib().ct_census_stream_timer_start(self._h))

    def timer_stop(self) -> float:
        ms = C.c_float()
        check(lib().ct_census_stream_timer_stop(self._h, C.byref(ms)))
        return ms.value


class ConfNet(_Driver):
    """Learned confidence net over census cost curves (ct_confnet_*)."""
    _create = "ct_confnet_create"

    def configure(self, device: int, max_batch: int):
        check(lib().ct_confnet_configure(self._h, device, max_batch))

    def init(self, seed: int):
        check(lib().ct_confnet_init(self._h, seed))

    def set_params(self, params):
        import numpy as np
        p = np.ascontiguousarray(params, np.float32)
        check(lib().ct_confnet_set_params(self._h, p.ctypes.data, p.size))

    def get_params(self):
        import numpy as np
        p = np.empty(CT_CONFNET_PARAMS, np.float32)
        check(lib().ct_confnet_get_params(self._h, p.ctypes.data, p.size))
        return p

    def gather(self, samples, curves: "CurveVolume", disp, xy, stream=None):
        """samples: (n, 128) uint8 CUDA tensor of re-centred curves; disp: the
        winner map (uint8 / int16); xy: (n, 2) int32 CUDA tensor."""
        check(lib().ct_confnet_gather(self._h, samples.data_ptr(), C.byref(curves.desc()), _img_ref(disp),
                                      xy.data_ptr(), xy.shape[0], _stream(stream)))

    def loss_grad(self, samples, labels, grad=None, loss=None, stream=None):
        check(lib().ct_confnet_loss_grad(self._h, samples.data_ptr(), labels.data_ptr(), samples.shape[0],
                                         None if grad is None else grad.data_ptr(),
                                         None if loss is None else loss.data_ptr(), _stream(stream)))

    def train_step(self, samples, labels, lr: float, loss=None, stream=None):
        check(lib().ct_confnet_train_step(self._h, samples.data_ptr(), labels.data_ptr(), samples.shape[0], lr,
                                          None if loss is None else loss.data_ptr(), _stream(stream)))

    def scores(self, out, samples, stream=None):
        check(lib().ct_confnet_scores(self._h, out.data_ptr(), samples.data_ptr(), samples.shape[0],
                                      _stream(stream)))

    def infer(self, score, curves: "CurveVolume", disp, checked=None, threshold: float = 0.5, stream=None):
        """Score map (float32, may be None) of a curve volume; disp: its winner
        map; checked (optional, same dtype as disp): disp with disparities
        scoring below threshold marked invalid, as the cross-check marks them."""
        check(lib().ct_confnet_infer(self._h, _img_ref(score), C.byref(curves.desc()), _img_ref(disp),
                                     _img_ref(checked), threshold, _stream(stream)))


def census_match_static(disp, left, right, disp_count: int, left_to_right: bool = True, device_status=None,
                        stream=None):
    """ct_bm_census_process_static: census matching with no device allocation
    (static scratch; images up to 2,097,152 pixels with rows rounded up to a
    multiple of 4). Without device_status, timeouts go to the static word
    that census_static_status() reads."""
    st = None if device_status is None else C.c_void_p(device_status.data_ptr())
    check(lib().ct_bm_census_process_static(_img_ref(disp), _img_ref(left), _img_ref(right), disp_count,
                                            int(left_to_right), st, _stream(stream)))


def census_static_status() -> int:
    """ct_bm_census_static_status: reads and clears the static status word of
    census_match_static calls made without a device_status (synchronises)."""
    v = C.c_int32()
    check(lib().ct_bm_census_static_status(C.byref(v)))
    return v.value


_synth = None


def synth_lib() -> C.CDLL:
    """Loads libctsynth.so, the host-only generator library (not the matcher)."""
    global _synth
    if _synth is None:
        if not SYNTH_PATH.exists():
            raise ImportError(f"{SYNTH_PATH} not built: run python module.clutec.cuda_b200/build.py")
        _synth = C.CDLL(str(SYNTH_PATH))
        _synth.ct_synth_pair.argtypes = [C.c_int32, C.c_uint64, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_void_p]
        _synth.ct_synth_pair.restype = C.c_int
    return _synth


def synth_pair(kind: int, seed: int, width: int, height: int, dmax: int):
    """Seeded synthetic pair -> (left u8, right u8, gt int16, occ u8) numpy
    arrays, from libctsynth.so (ct_synth_pair, include/ctsynth.h)."""
    import numpy as np
    L = np.empty((height, width), np.uint8)
    R = np.empty((height, width), np.uint8)
    G = np.empty((height, width), np.int16)
    O = np.empty((height, width), np.uint8)
    rc = synth_lib().ct_synth_pair(kind, seed, width, height, dmax, L.ctypes.data, R.ctypes.data,
                                   G.ctypes.data, O.ctypes.data)
    if rc != CT_OK:
        raise CtError(rc, f"ct_synth_pair: bad arguments (kind {kind}, {width}x{height}, dmax {dmax})")
    return L, R, G, O


def probe_pipe_rates(device: int = 0) -> dict:
    r = ct_pipe_rates()
    check(lib().ct_probe_pipe_rates(device, C.byref(r)))
    return {k: getattr(r, k) for k, _ in ct_pipe_rates._fields_ if k != "reserved"}
