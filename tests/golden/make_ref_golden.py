"""Writes tests/golden/ref_pin.npz: outputs of the reference's own census
transform and cross-check kernels (oracle/_ref/libctref.so, built from the
reference sources by oracle/ref/build_ref.py) on seeded inputs, so that the
oracle stays pinned to the reference where the reference is not present.

    python tests/golden/make_ref_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))

# census sizes: (W - 2) % 8 == 0 and (H - 2) % 16 == 0 where the reference
# driver's grid misses the last interior column / row, and ragged ones
CENSUS_SIZES = [(10, 18), (37, 23), (64, 48), (130, 66), (3, 3), (8, 9)]
# cross-check: (W, H, D, tol, left_to_right)
CC_CASES = [(37, 23, 8, 1, 1), (40, 19, 6, 0, 0), (33, 35, 4, 2, 1), (20, 20, 3, 12, 1), (66, 17, 12, 1, 0)]


def census_input(rng, W, H):
    img = rng.integers(0, 256, (H, W), dtype=np.uint8)
    img[::3, ::2] = 128  # ties with the centre (strict compare)
    return img


def code_map(rng, W, H, D):
    """Disparity codes 1..D with Unknown (0), CannotEvaluate, Inconsistent,
    NotSpecific and Last mixed in."""
    c = rng.integers(1, D + 1, (H, W)).astype(np.uint16)
    m = rng.random((H, W))
    c[m < 0.05] = 0xFFFF
    c[(m >= 0.05) & (m < 0.09)] = 0
    c[(m >= 0.09) & (m < 0.11)] = 0xFFFA
    c[(m >= 0.11) & (m < 0.12)] = 0xFFFC
    c[(m >= 0.12) & (m < 0.13)] = 0xFFEF
    return c


ARRAY_SUM_PATCHES = [(3, 3), (5, 5), (9, 9), (11, 11), (16, 16), (9, 5)]


def array_sum_expected(oracle, px, py, dims, tile):
    """What the reference's AlgoArraySum_W32H16<128, px, py> delivers for each
    of Sum, SumCache, SumCache3, built from the oracle's box sums: (3 modes,
    3 planes, PatchCountY, DataArraySizeX), -1 where nothing is delivered."""
    sx, sy, pcx, pcy, _ = dims
    t = tile.astype(np.int32)
    out = np.full((3, 3, pcy, sx), -1, np.int32)
    for mode in range(3):
        chans = [t, t * t, 3 * t + 1] if mode == 2 else [t]
        for c, ch in enumerate(chans):
            out[mode, c, :, :pcx] = oracle.box_sums(ch, px, py)[:pcy, :pcx]
    return out


def digest(a) -> str:
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a, np.int32).tobytes()).hexdigest()


def make(seed: int = 2024) -> dict:
    import ref_lib
    rng = np.random.default_rng(seed)
    out = {}
    for k, (px, py) in enumerate(ARRAY_SUM_PATCHES):
        dims = ref_lib.array_sum_dims(px, py)
        tile = rng.integers(0, 256, (dims[1], dims[0])).astype(np.uint8)
        res = np.stack([ref_lib.array_sum(px, py, mode, tile) for mode in range(3)])
        out[f"asum{k}_tile"] = tile
        out[f"asum{k}_par"] = np.array([px, py, *dims], np.int32)
        out[f"asum{k}_sha256"] = np.array(digest(res))
    for k, (W, H) in enumerate(CENSUS_SIZES):
        img = census_input(rng, W, H)
        out[f"census{k}_in"] = img
        out[f"census{k}_out"] = ref_lib.census3x3(img, fill=0xAB)
    for k, (W, H, D, tol, lr) in enumerate(CC_CASES):
        a, b = code_map(rng, W, H, D), code_map(rng, W, H, D)
        init = rng.integers(0, 65536, (H, W)).astype(np.uint16)
        res, (mn, mx) = ref_lib.crosscheck(a, b, tol, lr, init)
        out[f"cc{k}_lr"], out[f"cc{k}_rl"], out[f"cc{k}_init"] = a, b, init
        out[f"cc{k}_out"] = res
        out[f"cc{k}_range"] = np.array([mn, mx], np.int32)
        out[f"cc{k}_par"] = np.array([tol, lr], np.int32)
    return out


if __name__ == "__main__":
    dst = ROOT / "tests" / "golden" / "ref_pin.npz"
    np.savez_compressed(dst, **make())
    print(dst, dst.stat().st_size, "bytes")
