"""The reference-compat restatement (oracle/compat.cpp) on the CPU: known
answers on an exact shift, a second brute-force restatement of every
method's scan and ID rules (pure Python loops on small images, following the
reference lines each step cites), and the thresholds of the GPU parity cases
reaching every ID rule."""
import numpy as np
import pytest

from test_compat_gpu import CASES, IDS

FIRST, LAST, CANNOT, SAT, NOTFOUND, NOTSPEC = 1, 0xFFEF, 0xFFFF, 0xFFFE, 0xFFFD, 0xFFFC


def shifted_pair(W=120, H=60, K=7, seed=1):
    rng = np.random.default_rng(seed)
    L = rng.integers(0, 256, (H, W), dtype=np.uint8)
    R = np.empty_like(L)
    R[:, :W - K] = L[:, K:]  # L(x) = R(x - K)
    R[:, W - K:] = rng.integers(0, 256, (H, K))
    return L, R, K


@pytest.mark.parametrize("method,patch,score,y", [("sad1", 9, 1e9, 0), ("sad1", 16, 1e9, 0), ("ncc", 11, 0.0, 255),
                                                  ("aw1", 3, 0.0, 65535), ("aw2", 5, 1e9, 0), ("bm1", 9, 0.0, 49087)])
def test_exact_shift_known_answers(oracle, method, patch, score, y):
    L, R, K = shifted_pair()
    out = oracle.compat_match(L, R, method, 32, patch, score_thresh=score)
    inner = out[15:-15, 40:-20]
    assert (inner[..., 0] == FIRST + K).all()
    if method == "ncc":  # FP32 means / deviations: a perfect match rounds to 254 or 255
        assert (inner[..., 1] >= 254).all() and (inner[..., 1] == 255).mean() > 0.5
    else:
        assert (inner[..., 1] == y).all()
    # right-to-left: base = right image, match column x + d
    out = oracle.compat_match(L, R, method, 32, patch, score_thresh=score, left_to_right=False)
    assert (out[15:-15, 20:-40, 0] == FIRST + K).all()


def test_gpu_case_thresholds_reach_every_id(ct, oracle):
    seen = set()
    for method, patch, sim, lr, dmin, grad, score, delta in CASES:
        W, H, D = 157, 71, 40
        L, R, _, _ = ct.synth_pair(1 + (patch % 3 == 0), 3 * patch + dmin + sim, W, H, dmin + D - 1)
        x = oracle.compat_match(L, R, method, D, patch, dmin=dmin, sim_type=sim, left_to_right=lr,
                                grad_thresh=grad, score_thresh=score, min_delta_thresh=delta)[..., 0]
        seen |= {k for k, v in IDS.items() if (x == v).any()}
        seen |= {"disparity"} if ((x >= 1) & (x <= LAST)).any() else set()
    assert seen == set(IDS) | {"disparity"}


# ---- second restatement, pure Python -------------------------------------------

f32 = np.float32


def _sp(a, b, scale):
    f1 = f32(2.0) * (f32(a) / f32(255.0) - f32(0.5))
    f2 = f32(2.0) * (f32(b) / f32(255.0) - f32(0.5))
    return int(f32(f32(f1 * f2) * f32(scale)))


def _brute(L, R, method, D, patch, dmin, sim, lr, grad, score, delta):
    H, W = L.shape
    B, M = (L, R) if lr else (R, L)
    B, M = B.astype(np.int64), M.astype(np.int64)
    aw = method in ("aw1", "aw2")
    s = patch
    P = 3 * s if aw else patch
    a, b = P // 2, P - 1 - P // 2
    n = 3 * s * s if aw else P * P
    out = np.zeros((H, W, 4), np.uint16)
    Bx = np.concatenate([B, np.zeros((H, 1), np.int64)], 1)  # zero column beyond the edge

    def box(img, x0, y0, w, h):
        return int(img[y0:y0 + h, x0:x0 + w].sum())

    def sim_val(p, q):
        if method in ("sad1", "aw2"):
            return abs(p - q)
        if method == "ncc":
            return p * q
        if method == "aw1":
            return _sp(p, q, 255.0) if sim else 255 - abs(p - q)
        return _sp(p, q, 127.0) if sim else (255 - abs(p - q)) >> 1

    def score_at(x, y, d):
        xm = x - d if lr else x + d
        e = np.zeros((H, W), np.int64)
        for yy in range(max(0, y - P), min(H, y + P)):
            for xx in range(max(0, x - P), min(W, x + P)):
                xq = xm + (xx - x)
                if 0 <= xq < W:
                    e[yy, xx] = sim_val(int(B[yy, xx]), int(M[yy, xq]))
        if not aw:
            return box(e, x - a, y - a, P, P), xm
        sub = lambda cx, cy: box(e, cx - s // 2, cy - s // 2, s, s)  # noqa: E731
        nb = sorted([sub(x, y - s), sub(x - s, y), sub(x, y + s), sub(x + s, y)])
        return (sub(x, y) + nb[3] + nb[2] if method == "aw1" else sub(x, y) + nb[0] + nb[1]), xm

    def gate(x, y):
        if grad <= 0:
            return False
        g = np.abs(Bx[:, :-1] - Bx[:, 1:])
        if method in ("sad1", "ncc"):
            return f32(box(g, x - a, y - a, P, P)) / f32(P * P) < f32(grad)
        if method in ("bm1", "aw1"):
            fm = f32(box(B, x - a, y - a, P, P)) / f32(P * P)
            fm2 = f32(box(B * B, x - a, y - a, P, P)) / f32(P * P)
            sd = f32(np.sqrt(abs(f32(fm2 - f32(fm * fm)))))
            sd = f32(f32(f32(int(sd)) / f32(255)) * f32(100)) if method == "aw1" else f32(f32(sd / f32(255)) * f32(100))
            return sd < f32(grad)
        sub = lambda cx, cy: box(g, cx - s // 2, cy - s // 2, s, s)  # noqa: E731
        nb = sorted([sub(x, y - s), sub(x - s, y), sub(x, y + s), sub(x + s, y)])
        return f32(sub(x, y) + nb[0] + nb[1]) / f32(n) < f32(grad)

    def ncc_u8(x, y, S, xm):
        fBm = f32(box(B, x - a, y - a, P, P)) / f32(P * P)
        fBs = f32(np.sqrt(f32(f32(box(B * B, x - a, y - a, P, P)) / f32(P * P)) - f32(fBm * fBm)))
        fT = f32(box(M, xm - a, y - a, P, P)) / f32(P * P)
        fT2 = f32(box(M * M, xm - a, y - a, P, P)) / f32(P * P)
        fTs = f32(np.sqrt(f32(fT2 - f32(fT * fT))))
        norm = f32(fBs * fTs)
        v = f32(0.0) if not norm >= f32(1.0) else f32(f32(f32(S) / f32(P * P)) - f32(fBm * fT)) / norm
        v = v if v > 0 else f32(0.0)
        return int(min(f32(255.0), f32(v * f32(255.0))))

    def s2f(v):
        return f32(f32(v) / f32(n)) * f32(f32(100.0) / f32(255))

    def f2u(f):
        t = f32(f32(f32(f / f32(100.0)) + f32(1.0)) / f32(2.0))
        return int(f32(min(max(t, f32(0)), f32(1)) * f32(65535)))

    for y in range(H):
        for x in range(W):
            if not (x - a >= 0 and x + b < W and y - a >= 0 and y + b < H):
                out[y, x] = (CANNOT, 0, 0, 0)
                continue
            search = lambda d: (x - d - a >= 0) if lr else (x + d + b <= W - 1)  # noqa: E731
            disp = CANNOT if gate(x, y) else 0
            if method in ("ncc", "aw1", "bm1"):
                st = dict(p2=0, p=0, mx=0 if method == "ncc" else -32767, n=0, n2=0, last=0)
                for d in range(dmin, dmin + D):
                    if not search(d) or disp > LAST:
                        continue
                    S, xm = score_at(x, y, d)
                    v = ncc_u8(x, y, S, xm) if method == "ncc" else int(np.int16(S))
                    code = d + FIRST
                    above = v > st["mx"]
                    jb, j2b = (not above and disp + 1 == code), (not above and disp + 2 == code)
                    if above:
                        st.update(p2=st["p"], p=st["last"], mx=v, n=v, n2=v)
                        disp = code
                    if jb:
                        st["n"] = v
                    if j2b:
                        st["n2"] = v
                    st["last"] = v
                if disp > LAST or disp == 0:
                    out[y, x] = (disp, 0, 0, 0)
                    continue
                sat = disp - FIRST <= dmin + 1 or disp - FIRST >= dmin + D - 1
                if method == "ncc":
                    d1 = max(abs(st["p"] - st["mx"]), abs(st["p2"] - st["mx"]))
                    d2 = max(abs(st["n"] - st["mx"]), abs(st["n2"] - st["mx"]))
                    if f32(st["mx"]) / f32(255) >= f32(score):
                        ident = SAT if sat else (disp if d1 >= int(delta) and d2 >= int(delta) else NOTSPEC)
                    else:
                        ident = NOTFOUND
                    out[y, x] = (ident, st["mx"], d1, d2)
                else:
                    fm = s2f(st["mx"])
                    fdp = max(abs(s2f(st["p"]) - fm), abs(s2f(st["p2"]) - fm))
                    fdn = max(abs(s2f(st["n"]) - fm), abs(s2f(st["n2"]) - fm))
                    spec = fdp >= f32(delta) and fdn >= f32(delta)
                    ident = (SAT if sat else (disp if spec else NOTSPEC)) if fm >= f32(score) else NOTFOUND
                    out[y, x] = (ident, f2u(fm), f2u(fdp), f2u(fdn))
            else:
                mr = [0xFFFF, 0, 0, 0]  # x, y, z, w
                dmax = dmin + D - 1
                aw2 = method == "aw2"

                def upd(idx, inc):
                    nonlocal disp
                    if (disp > LAST) if aw2 else (disp == CANNOT):
                        return
                    v, _ = score_at(x, y, dmax - idx)
                    fmin = f32(v) / f32(n)
                    if idx == 0:
                        mr[3] = v
                        mr[1] = v
                        if aw2:
                            mr[2] = v
                    if v < mr[0] and fmin < f32(score):
                        mr[1], mr[0], mr[2], disp = mr[3], v, v, idx
                    elif disp + inc == idx:
                        mr[2] = v
                    mr[3] = v
                if aw2:
                    for idx in range(D):
                        if search(dmax - idx):
                            upd(idx, 1)
                else:
                    for idx in range(0, D, 4):
                        if search(dmax - idx):
                            upd(idx, 4)
                    for idx in range(D):
                        if search(dmax - idx) and idx + 4 >= disp and idx <= disp + 4:
                            upd(idx, 1)
                if disp > LAST:
                    out[y, x] = (disp, 0, 0, 0)
                    continue
                d1, d2 = abs(mr[1] - mr[0]), abs(mr[2] - mr[0])
                sat = (disp <= FIRST + 4 or disp >= FIRST + D - 4) if aw2 else (disp <= FIRST + 1 or disp >= FIRST + D - 1)
                spec = (d1 >= int(delta) and d2 >= int(delta)) if aw2 else (d1 > int(delta) and d2 > int(delta))
                if f32(mr[0]) / f32(n) < f32(score):
                    ident = FIRST + dmax - disp if (spec and not sat) else (SAT if sat else NOTSPEC)
                else:
                    ident = NOTFOUND
                out[y, x] = (ident, mr[0] // n, d1, d2)
    return out


@pytest.mark.parametrize("case", [c for c in CASES if c[1] <= 11])
def test_second_restatement_agrees(ct, oracle, case):
    method, patch, sim, lr, dmin, grad, score, delta = case
    W, H, D = 40, 33, 7
    L, R, _, _ = ct.synth_pair(1 + (patch % 3 == 0), 3 * patch + dmin + sim, W, H, dmin + D - 1)
    want = _brute(L, R, method, D, patch, dmin, sim, lr, grad, score, delta)
    got = oracle.compat_match(L, R, method, D, patch, dmin=dmin, sim_type=sim, left_to_right=lr,
                              grad_thresh=grad, score_thresh=score, min_delta_thresh=delta)
    np.testing.assert_array_equal(got, want)


def test_constant_divisor_quotient_is_ieee_exhaustive(oracle):
    """The reference-compat kernel divides integer-valued sums by the patch
    element count (and pixel values by 255) with a multiply by the rounded
    reciprocal and one remainder correction instead of an IEEE division; for
    every divisor it uses and every integer numerator up to 2^24 in magnitude
    the quotient equals the IEEE binary32 quotient."""
    divisors = sorted({p * p for p in range(1, 17)} | {3 * s * s for s in range(1, 6)} | {255})
    bad = {d: oracle.div_int_mismatches(d) for d in divisors}
    assert all(v == 0 for v in bad.values()), bad
