"""The CPU oracle against the golden fixtures and hand-computed answers.

The fixtures come from an independent brute-force restatement
(tests/golden/make_golden.py); agreement pins the oracle before it is used as
the checker of the CUDA kernels.
"""
import json

import numpy as np
import pytest

from conftest import GOLDEN


def load(name):
    return np.load(GOLDEN / name)


def test_census3x3_golden(oracle):
    g = load("census3x3.npz")
    out = oracle.census3x3(g["img"])
    H, W = g["img"].shape
    np.testing.assert_array_equal(out[1:H - 1, 1:W - 1], g["out"][1:H - 1, 1:W - 1])


def test_census3x3_leaves_border_unwritten(oracle):
    img = np.random.default_rng(0).integers(0, 256, (9, 11), dtype=np.uint8)
    out = oracle.census3x3(img, fill=0xAB)
    assert (out[0] == 0xAB).all() and (out[-1] == 0xAB).all()
    assert (out[:, 0] == 0xAB).all() and (out[:, -1] == 0xAB).all()


def test_census9x7_golden(oracle):
    g = load("census9x7.npz")
    np.testing.assert_array_equal(oracle.census9x7(g["img"]), g["out"])


def test_census9x7_known_patch(oracle):
    k = json.loads((GOLDEN / "known.json").read_text())["census9x7_patch"]
    img = np.array(k["patch"], np.uint8)
    out = oracle.census9x7(img)
    assert int(out[3, 4]) == int(k["descriptor"])
    # bit 63 and the centre bit (31) are never set
    assert int(out[3, 4]) >> 63 == 0 and (int(out[3, 4]) >> 31) & 1 == 0


@pytest.mark.parametrize("lr", [True, False])
def test_census_match_golden(oracle, lr):
    g = load("census_match.npz")
    d, c = oracle.match_census(g["L"], g["R"], int(g["D"]), 2, lr)
    tag = "lr" if lr else "rl"
    np.testing.assert_array_equal(d, g["disp_" + tag])
    valid = g["disp_" + tag] >= 0
    np.testing.assert_array_equal(c[valid], g["cost_" + tag][valid])


def test_census_match_on_descriptors_equals_image_path(oracle):
    g = load("census_match.npz")
    cl, cr = oracle.census9x7(g["L"]), oracle.census9x7(g["R"])
    d1, _ = oracle.match_census_desc(cl, cr, int(g["D"]))
    d2, _ = oracle.match_census(g["L"], g["R"], int(g["D"]))
    np.testing.assert_array_equal(d1, d2)


def test_sad_golden(oracle):
    g = load("sad.npz")
    d, c = oracle.match_sad(g["L"], g["R"], int(g["D"]), 4)
    np.testing.assert_array_equal(d, g["disp"])
    valid = g["disp"] >= 0
    np.testing.assert_array_equal(c[valid], g["cost"][valid])


def test_aw_golden(oracle):
    g = load("aw.npz")
    d, c, s32, s64 = oracle.match_aw(g["L"], g["R"], int(g["D"]))
    np.testing.assert_array_equal(d, g["disp"])
    valid = g["disp"] >= 0
    np.testing.assert_array_equal(c[valid], g["cost"][valid])
    np.testing.assert_allclose(s64[valid], g["sub"][valid], rtol=0, atol=1e-12)
    assert np.abs(s32[valid] - s64[valid]).max() <= 1e-4


def test_ncc_golden(oracle):
    g = load("ncc.npz")
    d, s32, s64 = oracle.match_ncc(g["L"], g["R"], int(g["D"]), 5)
    np.testing.assert_array_equal(d, g["disp"])
    valid = g["disp"] >= 0
    np.testing.assert_allclose(s64[valid], g["score"][valid], rtol=0, atol=1e-12)
    assert np.abs(s32[valid] - s64[valid]).max() <= 1e-4
    # the flat patch hits the sigma < 1 rule: score 0 at its interior pixels
    assert (s64[6, 6:9] == 0).all() and (s32[6, 6:9] == 0).all()


def test_crosscheck_golden(oracle):
    g = load("crosscheck.npz")
    out, (lo, hi) = oracle.crosscheck(g["base"], g["other"], 1)
    np.testing.assert_array_equal(out, g["out"])
    kept = g["out"][g["out"] >= 0]
    assert (lo, hi) == (int(kept.min()), int(kept.max()))


def test_constant_image_gives_lowest_d(oracle):
    img = np.full((30, 40), 91, np.uint8)
    d, _ = oracle.match_census(img, img, 8)
    assert (d[d >= 0] == 0).all()
    d, _ = oracle.match_sad(img, img, 8, 4)
    assert (d[d >= 0] == 0).all()


def test_pure_shift_recovered(oracle):
    k = json.loads((GOLDEN / "known.json").read_text())["shift"]["k"]
    rng = np.random.default_rng(5)
    L = rng.integers(0, 256, (40, 64)).astype(np.uint8)
    R = np.roll(L, -k, axis=1)  # R(x) = L(x + k): left pixel x matches right x - k
    d, _ = oracle.match_census(L, R, 12)
    inner = d[8:-8, 24:-8]
    assert (inner == k).mean() > 0.98
    d, _ = oracle.match_sad(L, R, 12, 4)
    assert (d[8:-8, 24:-8] == k).mean() > 0.98


def test_validity_rules(oracle):
    rng = np.random.default_rng(2)
    L = rng.integers(0, 256, (20, 30)).astype(np.uint8)
    R = rng.integers(0, 256, (20, 30)).astype(np.uint8)
    d, _ = oracle.match_census(L, R, 16)
    H, W = L.shape
    assert (d[:2] == -1).all() and (d[H - 2:] == -1).all()
    assert (d[:, :2] == -1).all() and (d[:, W - 2:] == -1).all()
    xs = np.arange(W)[None, :].repeat(H, 0)
    v = d >= 0
    assert (d[v] <= xs[v] - 2).all()  # matched window stays inside
    d, _ = oracle.match_census(L, R, 16, left_to_right=False)
    v = d >= 0
    assert (d[v] <= (W - 1 - 2) - xs[v]).all()


def test_guide_ranges_known_answer(oracle):
    """Scale 2, two coarse hints: block (0, 0) covers coarse columns 0..7,
    block (0, 1) columns 8..15; the second block row has no hint."""
    coarse = np.full((16, 16), -1, np.int16)
    coarse[0, 0] = 3    # -> 6 at full resolution
    coarse[2, 5] = 1    # -> 2, same block: range [max(0, 2 - 4), 6 + 4]
    coarse[7, 9] = 10   # -> 20: range [16, 24]
    lo, hi = oracle.guide_ranges(coarse, 32, 32)
    assert (lo[:16, :16] == 0).all() and (hi[:16, :16] == 10).all()
    assert (lo[:16, 16:] == 16).all() and (hi[:16, 16:] == 24).all()
    assert (lo[16:] > hi[16:]).all()


def test_guided_ncc_is_the_argmax_over_the_guide_range(oracle):
    """The guided oracle against a direct restatement: per pixel, FP32 NCC
    from direct window sums for each d in its range, strict '>' argmax."""
    H, W, D, r = 24, 40, 12, 2
    rng = np.random.default_rng(3)
    L = rng.integers(0, 256, (H, W), dtype=np.uint8)
    R = np.roll(L, -4, axis=1)
    R[:, -4:] = rng.integers(0, 256, (H, 4), dtype=np.uint8)
    R = np.clip(R.astype(np.int32) + rng.integers(-6, 7, (H, W)), 0, 255).astype(np.uint8)
    coarse = np.where(rng.random((H // 2, W // 2)) < 0.3, -1, rng.integers(0, 6, (H // 2, W // 2))).astype(np.int16)
    coarse[6:, 10:] = -1  # a block without hints
    lo, hi = oracle.guide_ranges(coarse, W, H)
    got, s32, _ = oracle.match_ncc_guided(L, R, D, coarse, r)
    n = (2 * r + 1) ** 2
    want = np.full((H, W), -1, np.int16)
    for y in range(r, H - r):
        for x in range(r, W - r):
            a = L[y - r:y + r + 1, x - r:x + r + 1].astype(np.int64)
            best, bd = np.float32(-2), -1
            for d in range(D):
                if x - d - r < 0 or d < lo[y, x] or d > hi[y, x]:
                    continue
                b = R[y - r:y + r + 1, x - d - r:x - d + r + 1].astype(np.int64)
                sx, sy = a.sum(), b.sum()
                vx, vy = n * (a * a).sum() - sx * sx, n * (b * b).sum() - sy * sy
                num = n * (a * b).sum() - sx * sy
                sc = np.float32(0) if vx * vy < n ** 4 else \
                    np.float32(num) / np.sqrt(np.float32(vx) * np.float32(vy))
                if sc > best:
                    best, bd = sc, d
            want[y, x] = bd
    np.testing.assert_array_equal(got, want)
    assert (lo[16:, 32:] > hi[16:, 32:]).all() and (got[16:, 32:] == -1).all()  # the block without hints


def _brute_wta(cost, D, dmin, r, lr, valid_match):
    """Brute-force box-aggregated WTA over disparities dmin .. dmin + D - 1:
    cost(y, x, xm) per pixel, windows and searchability as the oracle
    defines them (ties to the lowest disparity)."""
    H, W = cost.shape[:2]
    out = np.full((H, W), -1, np.int16)
    for y in range(r, H - r):
        for x in range(r, W - r):
            best = None
            for d in range(dmin, dmin + D):
                xm = x - d if lr else x + d
                if not valid_match(xm):
                    continue
                c = sum(int(cost[y + dy, x + dx, d]) for dy in range(-r, r + 1) for dx in range(-r, r + 1))
                if best is None or c < best:
                    best, out[y, x] = c, d
    return out


@pytest.mark.parametrize("lr", [True, False])
@pytest.mark.parametrize("dmin", [0, 3, 7])
def test_min_disparity_sad_and_census_against_brute_force(oracle, lr, dmin):
    """A minimum disparity shifts the search to x -/+ (dmin + d) and the
    stored disparity to dmin + d (BlockMatcherNCC.cu:789-795)."""
    rng = np.random.default_rng(dmin * 2 + lr)
    W, H, D, r = 29, 13, 6, 1
    L = rng.integers(0, 256, (H, W), dtype=np.uint8)
    R = rng.integers(0, 256, (H, W), dtype=np.uint8)
    b, m = (L, R) if lr else (R, L)
    Dt = dmin + D
    sad = np.zeros((H, W, Dt), np.int64)
    cb, cm = oracle.census9x7(b), oracle.census9x7(m)
    ham = np.zeros((H, W, Dt), np.int64)
    for d in range(Dt):
        for x in range(W):
            xm = x - d if lr else x + d
            if 0 <= xm < W:
                sad[:, x, d] = np.abs(b[:, x].astype(int) - m[:, xm].astype(int))
                ham[:, x, d] = [bin(int(u) ^ int(v)).count("1") for u, v in zip(cb[:, x], cm[:, xm])]
    ok = lambda xm: xm - r >= 0 and xm + r < W  # noqa: E731
    np.testing.assert_array_equal(oracle.match_sad(L, R, D, r, lr, dmin=dmin)[0], _brute_wta(sad, D, dmin, r, lr, ok))
    got = oracle.match_census(L, R, D, r, lr, dmin=dmin)[0]
    np.testing.assert_array_equal(got, _brute_wta(ham, D, dmin, r, lr, ok))
