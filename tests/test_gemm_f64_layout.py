"""The FP64 DMMA GEMM's fragment layout (dnnf90_b200/csrc/gemm_f64.cu) on the CPU.

A warp's m8n8k4 products sum over the four k its lanes hold, and its 4 x 4
fragments cover its 32 x 32 tile whichever rows, columns and k each lane
takes; the kernel permutes them so that every shared load is 16 bytes.  This
emulates one block's k-block in each mode with the kernel's index formulas
and the m8n8k4 fragment rules (A: lane (r8, c4) holds row r8, k c4; B: lane
(r8, c4) holds k c4, column r8; D: lane (r8, c4) holds row r8, columns 2 c4
and 2 c4 + 1), and checks that
  - the fragments, written back through the kernel's epilogue mapping, give
    A @ B for the block (each (m, n) once, every k once);
  - every 16-byte fragment load stays inside its staged tile and the eight
    lanes of each 16-byte phase fall on eight distinct 16-byte bank groups.
"""
import numpy as np

BM, BN, BK = 64, 64, 16
SA_MK, SB_NK = BK + 2, BK + 2      # [m][k], [n][k] tiles
SA_KM, SB_KN = BM + 4, BN + 4      # [k][m], [k][n] tiles
WARPS = [(wm, wn) for wn in (0, 32) for wm in (0, 32)]
LANES = [(l >> 2, l & 3) for l in range(32)]   # (r8, c4)


def dt_row(k):
    return 4 * (k & 3) + (k >> 2)


def emulate(mode, A, B):
    """D[m][n] of one block's k-block: A is [BM][BK] (m, k), B is [BK][BN]."""
    D = np.full((BM, BN), np.nan)
    loads = []                     # (tile, word offset, lane) per 16-byte load
    for wm, wn in WARPS:
        acc = np.zeros((32, 4, 4, 2))          # [lane][i][j][2]
        for ks in range(4):
            # per fragment (i, j): D_frag[row][col] += sum_kk A_frag[row][kk] B_frag[kk][col]
            for i in range(4):
                for j in range(4):
                    af = np.zeros((8, 4))
                    bf = np.zeros((4, 8))
                    for lane, (r8, c4) in enumerate(LANES):
                        if mode == "dw":
                            k = 4 * ks + c4
                            m = wm + 16 * (i >> 1) + 2 * r8 + (i & 1)
                            n = wn + 16 * (j >> 1) + 2 * r8 + (j & 1)
                        else:
                            k = 4 * c4 + ks
                            m = wm + 8 * i + r8
                            n = (wn + 8 * j + r8 if mode == "fwd"
                                 else wn + 16 * (j >> 1) + 2 * r8 + (j & 1))
                        af[r8, c4] = A[m, k]
                        bf[c4, r8] = B[k, n]
                    prod = af @ bf                     # [row][col]
                    for lane, (r8, c4) in enumerate(LANES):
                        acc[lane, i, j, 0] += prod[r8, 2 * c4]
                        acc[lane, i, j, 1] += prod[r8, 2 * c4 + 1]
        # the 16-byte loads of a k-block (word offsets in doubles)
        for lane, (r8, c4) in enumerate(LANES):
            if mode == "dw":
                for ks in range(4):
                    for ii in range(2):
                        loads.append(("a", (4 * ks + c4) * SA_KM + wm + 16 * ii + 2 * r8, lane, (ks, ii)))
                    for jj in range(2):
                        loads.append(("b", (4 * ks + c4) * SB_KN + wn + 16 * jj + 2 * r8, lane, (ks, jj)))
            else:
                for h in range(2):
                    for i in range(4):
                        loads.append(("a", (wm + 8 * i + r8) * SA_MK + 4 * c4 + 2 * h, lane, (h, i)))
                    if mode == "fwd":
                        for j in range(4):
                            loads.append(("b", (wn + 8 * j + r8) * SB_NK + 4 * c4 + 2 * h, lane, (h, j)))
                    else:
                        for e in range(2):
                            for jj in range(2):
                                loads.append(("b", (4 * (2 * h + e) + c4) * SB_KN + wn + 16 * jj + 2 * r8,
                                              lane, (h, e, jj)))
        # the epilogue's mapping back to (m, n)
        for lane, (r8, c4) in enumerate(LANES):
            for i in range(4):
                if mode == "fwd":
                    m = wm + 8 * i + r8
                    for j in range(4):
                        n = wn + 8 * j + 2 * c4
                        for q in range(2):
                            assert np.isnan(D[m, n + q])
                            D[m, n + q] = acc[lane, i, j, q]
                else:
                    m = (wm + 16 * (i >> 1) + 2 * r8 + (i & 1) if mode == "dw"
                         else wm + 8 * i + r8)
                    for jj in range(2):
                        n = wn + 16 * jj + 4 * c4
                        vals = [acc[lane, i, 2 * jj, 0], acc[lane, i, 2 * jj + 1, 0],
                                acc[lane, i, 2 * jj, 1], acc[lane, i, 2 * jj + 1, 1]]
                        for q in range(4):
                            assert np.isnan(D[m, n + q])
                            D[m, n + q] = vals[q]
    return D, loads


def check_loads(mode, loads):
    size = {"fwd": {"a": BM * SA_MK, "b": BN * SB_NK},
            "dt": {"a": BM * SA_MK, "b": BK * SB_KN},
            "dw": {"a": BK * SA_KM, "b": BK * SB_KN}}[mode]
    for tile, off, lane, key in loads:
        assert off % 2 == 0 and 0 <= off and off + 2 <= size[tile], (mode, tile, off)
    # one 16-byte load instruction per (tile, key) and warp: its four 8-lane phases
    byinst = {}
    for tile, off, lane, key in loads:
        byinst.setdefault((tile, key), {}).setdefault(lane, []).append(off)
    for (tile, key), lanes in byinst.items():
        nwarps = len(next(iter(lanes.values())))
        for w in range(nwarps):
            for ph in range(4):
                slots = {(lanes[l][w] * 8 // 16) % 8 for l in range(ph * 8, ph * 8 + 8)}
                assert len(slots) == 8, (mode, tile, key, w, ph)


def test_fragments_cover_the_product_and_loads_are_conflict_free():
    rng = np.random.default_rng(5)
    for mode in ("fwd", "dt", "dw"):
        A = rng.standard_normal((BM, BK))
        B = rng.standard_normal((BK, BN))
        D, loads = emulate(mode, A, B)
        assert not np.isnan(D).any(), mode
        np.testing.assert_allclose(D, A @ B, rtol=1e-13, atol=1e-13)
        check_loads(mode, loads)


def test_dt_rows_are_a_permutation_of_the_k_block():
    assert sorted(dt_row(k) for k in range(BK)) == list(range(BK))
    # DT's lane (c4) at k-step ks reads row 4 ks + c4, which holds k = 4 c4 + ks
    for ks in range(4):
        for c4 in range(4):
            assert dt_row(4 * c4 + ks) == 4 * ks + c4
