"""Generates the golden fixtures in this directory.

The reference ships no tests or golden vectors, so these fixtures come from a
second, independent restatement of the matcher semantics written as plain
brute-force Python loops (direct window sums, no running sums, no shared code
with oracle/oracle.cpp), on small seeded inputs plus hand-constructed cases:

  census3x3.npz  reference 3x3 census (CensusTransform.cu:103-119)
  census9x7.npz  9x7 / 64-bit census
  census_match.npz  census + 5x5 Hamming box + WTA, both directions
  sad.npz        9x9 SAD + WTA (BlockMatcherSAD1 exhaustive mode)
  aw.npz         best-of-5 shifted 7x7 SAD windows + parabolic sub-pixel (FP64)
  ncc.npz        11x11 NCC with the sigma < 1 rule (BlockMatcherNCC.cu:255-262), FP64
  crosscheck.npz cross-check with tolerance 1 (CrossCheckDisparityMaps.cu:63-110)
  known.json     hand-computed answers: census of a single patch, constant
                 image -> d = 0, pure shift by k -> d = k in the interior.

Run: python tests/golden/make_golden.py  (takes under a minute)
"""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent


def rng_images(seed, W, H, shift_field=None, noise=4):
    r = np.random.default_rng(seed)
    L = r.integers(0, 256, size=(H, W), dtype=np.int64)
    # smooth a little so windows carry structure
    L = ((L + np.roll(L, 1, 1) + np.roll(L, 1, 0)) // 3).astype(np.int64)
    R = np.zeros_like(L)
    for y in range(H):
        for x in range(W):
            d = 0 if shift_field is None else shift_field[y][x]
            xs = x + d
            R[y][x] = L[y][xs] if 0 <= xs < W else r.integers(0, 256)
    R = np.clip(R + r.integers(-noise, noise + 1, size=R.shape), 0, 255)
    return L.astype(np.uint8), R.astype(np.uint8)


def census3x3(img):
    H, W = len(img), len(img[0])
    out = [[0] * W for _ in range(H)]
    order = [(-1, -1), (0, -1), (1, -1), (-1, 0), (1, 0), (-1, 1), (0, 1), (1, 1)]
    for y in range(1, H - 1):
        for x in range(1, W - 1):
            c = int(img[y][x])
            v = 0
            for i, (dx, dy) in enumerate(order):
                if int(img[y + dy][x + dx]) > c:
                    v |= 1 << (7 - i)
            out[y][x] = v
    return out


def census9x7(img):
    H, W = len(img), len(img[0])
    out = [[0] * W for _ in range(H)]
    for y in range(H):
        for x in range(W):
            if not (4 <= x < W - 4 and 3 <= y < H - 3):
                continue
            c = int(img[y][x])
            v = 0
            k = 0
            for dy in range(-3, 4):
                for dx in range(-4, 5):
                    if int(img[y + dy][x + dx]) > c:
                        v |= 1 << (62 - k)
                    k += 1
            out[y][x] = v
    return out


def wta(W, H, D, r, cost, lr=True):
    """Brute force: for each valid pixel, for d ascending, direct window sum."""
    disp = [[-1] * W for _ in range(H)]
    best = [[-1] * W for _ in range(H)]
    for y in range(r, H - r):
        for x in range(r, W - r):
            bc, bd = None, -1
            for d in range(D):
                xm = x - d if lr else x + d
                if xm - r < 0 or xm + r >= W:
                    continue
                c = 0
                for dy in range(-r, r + 1):
                    for dx in range(-r, r + 1):
                        c += cost(x + dx, y + dy, xm + dx)
                if bc is None or c < bc:
                    bc, bd = c, d
            disp[y][x], best[y][x] = bd, bc
    return disp, best


def census_match(L, R, D, lr=True):
    cl, cr = census9x7(L), census9x7(R)
    H, W = len(L), len(L[0])
    cb, cm = (cl, cr) if lr else (cr, cl)
    return wta(W, H, D, 2, lambda x, y, xm: bin(cb[y][x] ^ cm[y][xm]).count("1"), lr)


def sad(L, R, D, r=4):
    H, W = len(L), len(L[0])
    return wta(W, H, D, r, lambda x, y, xm: abs(int(L[y][x]) - int(R[y][xm])))


def aw(L, R, D):
    H, W = len(L), len(L[0])

    def S(x, y, d):
        return sum(abs(int(L[y + dy][x + dx]) - int(R[y + dy][x + dx - d]))
                   for dy in range(-3, 4) for dx in range(-3, 4))

    disp = [[-1] * W for _ in range(H)]
    cost = [[-1] * W for _ in range(H)]
    sub = [[-1.0] * W for _ in range(H)]
    for y in range(6, H - 6):
        for x in range(6, W - 6):
            A = []
            for d in range(D):
                if x - d - 6 < 0:
                    break
                A.append(min(S(x, y, d), S(x - 3, y, d), S(x + 3, y, d), S(x, y - 3, d), S(x, y + 3, d)))
            bd = min(range(len(A)), key=lambda i: (A[i], i))
            disp[y][x], cost[y][x] = bd, A[bd]
            s = float(bd)
            if 0 < bd < D - 1 and bd + 1 < len(A):
                cm, c0, cp = A[bd - 1], A[bd], A[bd + 1]
                den = cm - 2 * c0 + cp
                if den > 0:
                    s = bd + (cm - cp) / (2.0 * den)
            sub[y][x] = s
    return disp, cost, sub


def ncc(L, R, D, r=5):
    H, W = len(L), len(L[0])
    n = (2 * r + 1) ** 2
    disp = [[-1] * W for _ in range(H)]
    score = [[0.0] * W for _ in range(H)]
    for y in range(r, H - r):
        for x in range(r, W - r):
            a = [int(L[y + dy][x + dx]) for dy in range(-r, r + 1) for dx in range(-r, r + 1)]
            sx, sxx = sum(a), sum(v * v for v in a)
            vx = n * sxx - sx * sx
            best, bd = None, -1
            for d in range(D):
                if x - d - r < 0:
                    break
                b = [int(R[y + dy][x + dx - d]) for dy in range(-r, r + 1) for dx in range(-r, r + 1)]
                sy, syy = sum(b), sum(v * v for v in b)
                sxy = sum(p * q for p, q in zip(a, b))
                vy = n * syy - sy * sy
                num = n * sxy - sx * sy
                s = 0.0 if vx * vy < n ** 4 else num / math.sqrt(vx * vy)
                if best is None or s > best:
                    best, bd = s, d
            disp[y][x], score[y][x] = bd, best
    return disp, score


def crosscheck(base, other, tol=1):
    H, W = len(base), len(base[0])
    out = [[0] * W for _ in range(H)]
    for y in range(H):
        for x in range(W):
            d = base[y][x]
            if d < 0:
                out[y][x] = d
                continue
            xo = x - d
            if not (0 <= xo < W):
                out[y][x] = -2
                continue
            do = other[y][xo]
            out[y][x] = d if (do >= 0 and abs(do - d) <= tol) else -2
    return out


def main():
    # random field of integer disparities for matcher inputs (L(x) = R(x - d))
    def field(seed, W, H, dmax):
        r = np.random.default_rng(seed)
        f = np.full((H, W), r.integers(0, dmax + 1))
        for _ in range(3):
            x0, y0 = r.integers(0, W - 4), r.integers(0, H - 4)
            f[y0:y0 + r.integers(3, H // 2), x0:x0 + r.integers(3, W // 2)] = r.integers(0, dmax + 1)
        return f

    def pair(seed, W, H, dmax):
        f = field(seed, W, H, dmax)
        # build right so that L(x, y) ~ R(x - d(x, y), y)
        r = np.random.default_rng(seed + 1)
        L = r.integers(0, 256, size=(H, W))
        L = ((L + np.roll(L, 1, 1) + np.roll(L, 1, 0)) // 3)
        R = r.integers(0, 256, size=(H, W))
        for y in range(H):
            for x in range(W):
                xr = x - f[y][x]
                if 0 <= xr < W:
                    R[y][xr] = L[y][x]
        R = np.clip(R + r.integers(-3, 4, size=R.shape), 0, 255)
        return L.astype(np.uint8), R.astype(np.uint8)

    L, R = pair(11, 37, 23, 9)
    np.savez_compressed(OUT / "census3x3.npz", img=L, out=np.array(census3x3(L.tolist()), np.uint8))
    np.savez_compressed(OUT / "census9x7.npz", img=L,
                        out=np.array(census9x7(L.tolist()), dtype=np.uint64))

    L, R = pair(12, 41, 19, 10)
    dlr, clr = census_match(L.tolist(), R.tolist(), 12, True)
    drl, crl = census_match(L.tolist(), R.tolist(), 12, False)
    np.savez_compressed(OUT / "census_match.npz", L=L, R=R, D=12, disp_lr=np.array(dlr, np.int16),
                        cost_lr=np.array(clr, np.int32), disp_rl=np.array(drl, np.int16),
                        cost_rl=np.array(crl, np.int32))
    cc = crosscheck(dlr, drl, 1)
    np.savez_compressed(OUT / "crosscheck.npz", base=np.array(dlr, np.int16), other=np.array(drl, np.int16),
                        out=np.array(cc, np.int16))

    L, R = pair(13, 36, 20, 8)
    d, c = sad(L.tolist(), R.tolist(), 10, 4)
    np.savez_compressed(OUT / "sad.npz", L=L, R=R, D=10, disp=np.array(d, np.int16), cost=np.array(c, np.int32))

    L, R = pair(14, 34, 22, 7)
    d, c, s = aw(L.tolist(), R.tolist(), 9)
    np.savez_compressed(OUT / "aw.npz", L=L, R=R, D=9, disp=np.array(d, np.int16), cost=np.array(c, np.int32),
                        sub=np.array(s, np.float64))

    L, R = pair(15, 30, 16, 6)
    # a flat patch exercises the sigma < 1 rule
    L[0:16, 0:14] = 77
    d, s = ncc(L.tolist(), R.tolist(), 8, 5)
    np.savez_compressed(OUT / "ncc.npz", L=L, R=R, D=8, disp=np.array(d, np.int16), score=np.array(s, np.float64))

    # hand-computed known answers
    patch = [[0] * 9 for _ in range(7)]
    patch[0][0] = 200   # (-4,-3): bit 62
    patch[3][5] = 101   # (+1, 0): position 32 -> bit 30
    patch[6][8] = 255   # (+4,+3): position 62 -> bit 0
    patch[3][3] = 100   # (-1, 0): equal-or-less neighbours give 0
    for r_ in range(7):
        for c_ in range(9):
            if patch[r_][c_] == 0:
                patch[r_][c_] = 50
    patch[3][4] = 100   # centre
    expect = (1 << 62) | (1 << 30) | 1
    known = {
        "census9x7_patch": {"patch": patch, "descriptor": str(expect)},
        "constant_image": {"note": "all costs equal -> lowest d (0) wins", "d": 0},
        "shift": {"note": "right = left shifted by k -> d = k in the interior", "k": 5},
    }
    (OUT / "known.json").write_text(json.dumps(known, indent=1))
    print("fixtures written to", OUT)


if __name__ == "__main__":
    main()
