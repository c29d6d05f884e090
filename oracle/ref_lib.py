"""ctypes loader for oracle/_ref/libctref.so: the reference's own census
transform and cross-check kernels compiled for the host CPU
(oracle/ref/build_ref.py; the reference sources are read where they lie, at
build time).

TEST INFRASTRUCTURE ONLY: used by tests/ and tests/golden/make_ref_golden.py
to pin the oracle to the reference's code. Needs the reference sources to
build; a copy already built travels with the tree.
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

_DIR = Path(__file__).resolve().parent
LIB_PATH = _DIR / "_ref" / "libctref.so"
_lib = None


def available(ref_root: Path | None = None) -> bool:
    """True if the library is built or can be built from the reference sources."""
    if LIB_PATH.exists():
        return True
    sys.path.insert(0, str(_DIR / "ref"))
    import build_ref
    root = ref_root or build_ref.DEFAULT_REF
    return (root / "CluTec.Cuda.ImgProc/CensusTransform.cu").exists()


def build(ref_root: Path | None = None) -> Path:
    sys.path.insert(0, str(_DIR / "ref"))
    import build_ref
    return build_ref.build(ref_root or build_ref.DEFAULT_REF)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(LIB_PATH))
        vp, i = C.c_void_p, C.c_int
        _lib.ref_census3x3.argtypes = [vp, i, i, i, vp, i]
        _lib.ref_crosscheck.argtypes = [vp, vp, i, i, i, i, vp, vp]
        _lib.ref_array_sum.argtypes = [i, i, i, vp, vp, vp]
        _lib.ref_array_sum.restype = i
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def census3x3(img, fill=0):
    """The reference kernel with its driver's grid; pixels it does not write
    keep `fill`."""
    img = np.ascontiguousarray(img, np.uint8)
    H, W = img.shape
    out = np.full((H, W), fill, np.uint8)
    lib().ref_census3x3(_p(img), W, H, W, _p(out), W)
    return out


def crosscheck(lr_codes, rl_codes, tol, left_to_right, out_init):
    """The reference kernel and driver on uint16 code maps; pixels it does
    not write keep out_init. -> (out, (min code, max code))"""
    a = np.ascontiguousarray(lr_codes, np.uint16)
    b = np.ascontiguousarray(rl_codes, np.uint16)
    out = np.array(out_init, np.uint16, copy=True)
    H, W = a.shape
    rng = np.zeros(2, np.int32)
    lib().ref_crosscheck(_p(a), _p(b), W, H, tol, 1 if left_to_right else 0, _p(out), _p(rng))
    return out, (int(rng[0]), int(rng[1]))


ARRAY_SUM_PATCHES = [(3, 3), (5, 5), (7, 7), (9, 9), (11, 11), (16, 16), (9, 5)]


def array_sum_dims(px, py):
    """(DataArraySizeX, DataArraySizeY, PatchCountX, PatchCountY, ColGroupSizeX)
    of AlgoArraySum_W32H16<128, px, py>."""
    dims = np.zeros(5, np.int32)
    if lib().ref_array_sum(px, py, 0, None, None, _p(dims)) != 0:
        raise ValueError(f"patch {px}x{py} not instantiated")
    return tuple(int(v) for v in dims)


def array_sum(px, py, mode, tile):
    """The reference's block box sums on one data tile (DataArraySizeY x
    DataArraySizeX int32): mode 0 Sum, 1 SumCache, 2 SumCache3 (channels v,
    v*v, 3v+1). -> (3, PatchCountY, DataArraySizeX) int32, -1 where no
    result was delivered."""
    sx, sy, _, ny, _ = array_sum_dims(px, py)
    tile = np.ascontiguousarray(tile, np.int32)
    assert tile.shape == (sy, sx)
    out = np.zeros((3, ny, sx), np.int32)
    dims = np.zeros(5, np.int32)
    lib().ref_array_sum(px, py, mode, _p(tile), _p(out), _p(dims))
    return out
