"""The storage layout of the tensor-core DST passes (csrc/tc_dst.cu, tc_dst.h),
restated in float64 on the CPU: block order of the lines, uv form of the
positions, the half-length matrix A, the tiles (odd frequencies read the u half,
even ones the v half), the epilogue's mirror pairs (columns c and TN - 1 - c of
a tile), the natural-order lines into the last pass, and the FP64 scatter.
Without rounding, the four passes must reproduce the 2D DST-I solve
x = S(m * S(b)) of src/fluid.jl:145-166 (scipy's dstn type 1, the same
unnormalised RODFT00) to rounding level; an index slip anywhere breaks it."""
import numpy as np
import pytest
import scipy.fft as sf


def blk(i, P):
    """tc_blk: physical index of storage index i (0 for the padding slot)."""
    if i < P // 2:
        return 2 * i + 1
    c = i - P // 2
    if c < P // 4:
        return 2 * (c + 1)
    if c == P // 4:
        return 0
    return 2 * c


def uvj(s, P):
    """tc_uvj: the pair (j, P - j) held in uv slot s (0 .. P/2 - 1)."""
    return 2 * s + 1 if s < P // 4 else 2 * (s - P // 4 + 1)


def _solve_as_the_kernel(b, mult, P):
    H = TN = P // 2
    phys = np.array([blk(i, P) for i in range(P)])
    uj = np.array([uvj(s, P) for s in range(H)])
    # A[r][s] = 2 sin(pi k j / P), k = blk(r), j = uvj(s); zero rows at the padding
    # and zero at (even k, j = P/2)
    A = 2 * np.sin(np.pi * ((phys[:, None] * uj[None, :]) % (2 * P)) / P)
    A[phys == 0] = 0.0
    A[np.ix_(phys % 2 == 0, uj == H)] = 0.0
    # the first pass's lines: line l = row y = blk(l), slots in uv form
    X = np.zeros((P, P))
    bb = np.zeros((P + 1, P + 1))  # 1-based padded copy of b[y - 1][x - 1]
    bb[1:P, 1:P] = b
    for l in range(P):
        y = phys[l]
        if y == 0:
            continue
        a, c = bb[y, uj], bb[y, P - uj]
        X[l, :H] = np.where(uj == H, a, a + c)
        X[l, H:] = np.where(uj == H, 0.0, a - c)
    # multiplier table [kx storage][ky storage]
    kx, ky = phys[:, None], phys[None, :]
    M = np.where((kx > 0) & (ky > 0), mult[(ky - 1).clip(0), (kx - 1).clip(0)], 0.0)

    def tpass(X, epi):
        Y = np.zeros((P, P))
        out = np.zeros((P - 1, P - 1))
        for m0 in range(0, P, 128):
            koff = 0 if m0 < H else H
            rows = np.arange(m0, m0 + 128)
            for nt in range(2):
                n0 = nt * TN
                D = A[m0:m0 + 128] @ X[n0:n0 + TN, koff:koff + H].T
                if epi == "f64":
                    y = phys[rows]
                    x = np.arange(n0, n0 + TN)
                    keep_y, keep_x = y > 0, x < P - 1
                    out[np.ix_(y[keep_y] - 1, x[keep_x])] = D[np.ix_(keep_y, keep_x)]
                    continue
                if epi == "mult":
                    D = D * M[n0:n0 + TN, m0:m0 + 128].T
                c = np.arange(TN // 2)
                u = D[:, c] + D[:, TN - 1 - c]
                v = D[:, c] - D[:, TN - 1 - c]
                lines = rows
                if epi == "nat":
                    k = phys[rows]
                    lines = np.where(k == 0, P - 1, k - 1)
                Y[np.ix_(lines, nt * (TN // 2) + c)] = u
                Y[np.ix_(lines, H + nt * (TN // 2) + c)] = v
        return out if epi == "f64" else Y

    return tpass(tpass(tpass(tpass(X, "split"), "mult"), "nat"), "f64")


@pytest.mark.parametrize("P", [256])
def test_storage_maps_reproduce_the_solve(P):
    m = P - 1
    rng = np.random.default_rng(P)
    b = rng.normal(size=(m, m))  # [y][x]
    i = np.arange(1, P)
    lam = -2 * (np.cos(np.pi * i[None, :] / P) + np.cos(np.pi * i[:, None] / P) - 2)  # [ky][kx]
    mult = (1.0 / (4 * P * P)) / lam
    exact = sf.dstn(sf.dstn(b, type=1) * mult, type=1)
    got = _solve_as_the_kernel(b, mult, P)
    assert np.linalg.norm(got - exact) / np.linalg.norm(exact) < 1e-13


def test_block_order_pairs_mirror_indices():
    for P in (256, 512):
        phys = [blk(i, P) for i in range(P)]
        assert sorted(phys) == list(range(P))  # 1 .. P-1 once, and one padding slot
        TN = P // 2
        for nt in range(2):
            for c in range(TN // 2):
                j, jm = phys[nt * TN + c], phys[nt * TN + TN - 1 - c]
                assert jm == 0 or j + jm == P, (P, nt, c, j, jm)
                assert uvj(nt * (TN // 2) + c, P) == j
