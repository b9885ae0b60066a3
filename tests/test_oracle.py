"""CPU oracle pinned by hand-computed known answers and by an independent
pure-Python restatement on small cases.

The reference ships no golden vectors for this path (its tests only write
PNGs, LibThunderVision/tests/stereotest.cpp:9-74), so the oracle is pinned by:
  * literal values worked out by hand below from the cited reference lines;
  * the reference table's own geometry (pathCount, the stale-end coverage);
  * a second, independent restatement in numpy-float32 scalar loops.
"""
import math

import numpy as np
import pytest

INF = np.float32(np.inf)
f32 = np.float32


# ---------------------------------------------------------------- known answers
def test_bt_known_answers(orc):
    # 5x1 row; tdvision/birchfieldcost.cu:14-39, clamp-to-edge taps
    L = np.array([[10, 20, 30, 20, 10]], np.float32)
    R = np.array([[20, 30, 20, 10, 0]], np.float32)
    C = orc.bt_cost(L, R, 4)  # HWD: (1, 5, 4)
    assert C[0, 2, 1] == 0.0
    assert C[0, 2, 0] == 5.0
    assert C[0, 0, 0] == 5.0
    assert C[0, 4, 2] == 5.0
    assert C[0, 3, 3] == 0.0
    assert np.isinf(C[0, 1, 2]) and np.isinf(C[0, 0, 1])


def test_ncc_known_answers(orc):
    L = np.arange(1, 10, dtype=np.float32).reshape(3, 3)
    R = L - 1
    C = orc.ncc_cost(L, R, 2, radius=1)
    # exact values, and the float32 evaluation order 1 - dom/sqrt(ls*rs)
    assert C[1, 1, 0] == pytest.approx(1 - 240 / math.sqrt(285 * 204), abs=1e-7)
    assert C[1, 1, 1] == pytest.approx(1 - 207 / math.sqrt(285 * 156), abs=1e-7)
    assert C[1, 1, 0] == f32(1) - f32(240) / np.sqrt(f32(285) * f32(204))
    assert C[1, 1, 1] == f32(1) - f32(207) / np.sqrt(f32(285) * f32(156))
    assert np.isinf(C[1, 0, 1])


def test_ssd_known_answer(orc):
    L = np.zeros((3, 3), np.float32)
    L[1, 1] = 4
    R = np.zeros((3, 3), np.float32)
    C = orc.ssd_cost(L, R, 1, radius=1)
    assert C[1, 1, 0] == 16.0
    # window at (0,0) with clamp covers (1,1) once
    assert C[0, 0, 0] == 16.0


def _vol_3x1():
    C = np.array([[1, 4, 2], [3, 0, 5], [2, 2, 0]], np.float32).reshape(1, 3, 3)
    return C


def test_sgm_standard_known_answer(orc):
    # W=3, H=1, D=3, P1=1, P2=3 expanded by hand (H+ = [1,4,2],[3,1,6],[3,2,1];
    # H- = [2,4,3],[5,1,5],[2,2,0]; vertical and diagonal walks are single cells)
    C = _vol_3x1()
    g = np.zeros((1, 3), np.float32)
    d4, _, S4 = orc.sgm(C, g, 1, 3, paths=4)
    np.testing.assert_array_equal(S4[0], [[5, 16, 9], [14, 2, 21], [9, 8, 1]])
    np.testing.assert_array_equal(d4[0], [0, 1, 2])
    d8, dn8, S8 = orc.sgm(C, g, 1, 3, paths=8)
    np.testing.assert_array_equal(S8[0], [[9, 32, 17], [26, 2, 41], [17, 16, 1]])
    np.testing.assert_array_equal(dn8[0], np.array([0, 1, 2], np.float32) / np.float32(3))


def test_sgm_ref_cpu_start_assign(orc):
    # REF_CPU assigns S = C at every walk start (tdvision/semiglobalcpu.cpp:81):
    # on a one-row image every vertical walk starts (and ends) on its own cell,
    # so the later vertical walks overwrite the horizontal sums with C.
    C = _vol_3x1()
    g = np.zeros((1, 3), np.float32)
    d, _, S = orc.sgm(C, g, 1, 3, paths=4, semantics=orc.SEM_REF_CPU, table=orc.TABLE_REF)
    np.testing.assert_array_equal(S, C)
    np.testing.assert_array_equal(d[0], [0, 1, 2])


def test_dp_known_answer(orc):
    # A(1) = [4,1,7] codes [0,-1,0]; A(2) = [3,3,1] codes [+1,0,-1];
    # backtrack from d=2 at x=2: writes 1, 0, 0
    d, dn = orc.dp(_vol_3x1())
    np.testing.assert_array_equal(d[0], [0, 0, 1])


def test_wta_ties_and_nan(orc):
    V = np.array([[3, 1, 1, 2], [np.nan, 2, 2, 5], [np.inf] * 4, [np.nan] * 4],
                 np.float32).reshape(1, 4, 4)
    d, dn = orc.wta(V)
    np.testing.assert_array_equal(d[0], [1, 1, 0, 0])


def test_fastwta_known_answer(orc):
    L = np.zeros((1, 6), np.float32)
    L[0, 3] = 9
    R = np.zeros((1, 6), np.float32)
    R[0, 1] = 9
    d, _ = orc.fastwta(L, R, 4, radius=0)
    assert d[0, 3] == 2  # the only zero-cost match
    assert d[0, 0] == 0


# ---------------------------------------------------------------- path table
def test_path_table_geometry(orc):
    for W, H in [(384, 288), (288, 384), (5, 3), (3, 5), (4, 4), (1, 1), (1, 7), (7, 1)]:
        t = orc.path_table(W, H, orc.TABLE_REF)
        assert len(t) == W + H + 2 * (W + H - 1)  # tdvision/semiglobal.cu:62
        f = orc.path_table(W, H, orc.TABLE_FULL)
        np.testing.assert_array_equal(t[:, [0, 1, 4, 5, 6]], f[:, [0, 1, 4, 5, 6]])
        # forward walks stay inside the image in both tables
        for sx, sy, ex, ey, dx, dy, n in f:
            assert 0 <= sx < W and 0 <= sy < H
            assert 0 <= sx + (n - 1) * dx < W and 0 <= sy + (n - 1) * dy < H
            assert (ex, ey) == (sx + (n - 1) * dx, sy + (n - 1) * dy)


def _coverage(t, W, H):
    cov = {}
    for sx, sy, ex, ey, dx, dy, n in t:
        for x0, y0, ddx, ddy in ((sx, sy, dx, dy), (ex, ey, -dx, -dy)):
            c = cov.setdefault((int(ddx), int(ddy)), np.zeros((H, W), int))
            for k in range(n):
                c[y0 + k * ddy, x0 + k * ddx] += 1
    return cov


def test_ref_table_stale_ends(orc):
    # 384x288: the (-1,-1) and (1,-1) reverse walks miss (W-H)*H = 27648
    # pixels and retrace one diagonal W-H+1 = 97 times; portrait breaks (-1,-1)
    cov = _coverage(orc.path_table(384, 288, orc.TABLE_REF), 384, 288)
    for d in [(-1, -1), (1, -1)]:
        assert (cov[d] == 0).sum() == 27648 and cov[d].max() == 97
    for d in [(1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (-1, 1)]:
        assert (cov[d] == 1).all()
    cov = _coverage(orc.path_table(288, 384, orc.TABLE_REF), 288, 384)
    assert (cov[(-1, -1)] == 0).sum() == 27360 and cov[(-1, -1)].max() == 96
    cov = _coverage(orc.path_table(384, 288, orc.TABLE_FULL), 384, 288)
    assert all((c == 1).all() for c in cov.values())


# ------------------------------------------- independent pure-Python restatement
def py_table(W, H, ref):
    """tdvision/semiglobal.cu:116-230, written out again."""
    t = []
    for i in range(H):
        t.append([0, i, W - 1, i, 1, 0, W])
    for i in range(W):
        t.append([i, 0, i, H - 1, 0, 1, H])
    for i in range(W):
        ey = min(i, H - 1)
        t.append([W - 1 - i, 0, W - 1, ey, 1, 1, ey + 1])
    for i in range(H - 1):
        ex = min(H - 1 - (i + 1), W - 1)
        t.append([0, i + 1, ex, H - 1, 1, 1, ex + 1])
    for i in range(W):
        n = min(i + 1, H)
        t.append([i, 0, 0, n - 1, -1, 1, n])
    for i in range(H - 1):
        n = min(H - (i + 1), W)
        t.append([W - 1, i + 1, W - 1 - n + 1, i + 1 + n - 1, -1, 1, n])
    if not ref:
        for e in t:
            e[2] = e[0] + (e[6] - 1) * e[4]
            e[3] = e[1] + (e[6] - 1) * e[5]
    return t


def py_sgm(C, img, p1, p2, adjust, paths, ref_table, sem):
    H, W, D = C.shape
    S = np.zeros_like(C)
    p1, p2 = f32(p1), f32(p2)

    def fmin(a, b):
        return f32(np.fmin(a, b))

    def smin(a, b):
        return b if b < a else a

    def walk(x, y, dx, dy, n):
        last = [INF] * (D + 2)
        last_min = [INF] * D
        for z in range(D):
            c = C[y, x, z]
            S[y, x, z] = c if sem == 1 else f32(S[y, x, z] + c)
            last[z + 1] = f32(c + p1) if sem == 2 else c
            last_min[z] = c
        li = img[y, x]
        for _ in range(1, n):
            x += dx
            y += dy
            if sem == 1:
                m = INF
                for z in range(D - 1):
                    m = fmin(last[z + 1], m)
            elif sem == 2:
                m = INF
                for z in range(D):
                    m = fmin(m, last_min[z])
            else:
                m = INF
                for z in range(D):
                    m = fmin(m, last[z + 1])
            I = img[y, x]
            pa = f32(p2 / f32(abs(f32(I - li)))) if adjust else p2
            li = I
            mp2 = f32(m + pa)
            new = [INF] * (D + 2)
            for z in range(D):
                a, b, e = last[z + 1], f32(last[z] + p1), f32(last[z + 2] + p1)
                if sem == 1:
                    mn = smin(a, smin(b, smin(e, mp2)))
                else:
                    mn = fmin(a, fmin(b, fmin(e, mp2)))
                v = f32(f32(C[y, x, z] + mn) - m)
                S[y, x, z] = f32(S[y, x, z] + v)
                new[z + 1] = v
                last_min[z] = v
            last = new

    for sx, sy, ex, ey, dx, dy, n in py_table(W, H, ref_table):
        if paths == 4 and dx != 0 and dy != 0:
            continue
        walk(sx, sy, dx, dy, n)
        walk(ex, ey, -dx, -dy, n)
    return S


@pytest.mark.parametrize("W,H,D", [(5, 3, 4), (3, 5, 3), (4, 4, 2), (6, 2, 3), (1, 4, 2), (4, 1, 1)])
@pytest.mark.parametrize("sem", [0, 1, 2])
def test_oracle_vs_python_restatement(orc, W, H, D, sem):
    rng = np.random.default_rng(W * 100 + H * 10 + D + sem)
    Li = rng.integers(0, 256, size=(H, W)).astype(np.float32) / np.float32(255)
    Ri = rng.integers(0, 256, size=(H, W)).astype(np.float32) / np.float32(255)
    C = orc.bt_cost(Li, Ri, D)
    for table in (0, 1):
        for adjust in (0, 1):
            for paths in (4, 8):
                p1, p2 = f32(30) / f32(255), f32(150) / f32(255)
                _, _, S = orc.sgm(C, Li, p1, p2, p2_mode=adjust, paths=paths, table=table,
                                  semantics=sem)
                Sp = py_sgm(C, Li, p1, p2, adjust, paths, table == 1, sem)
                np.testing.assert_array_equal(S, Sp)


def test_oracle_threads_match_sequential(orc):
    from thundervision_b200 import synthetic as syn
    L, R, _, _ = syn.pair_small(3)
    Lf, Rf = orc.u8_to_f32(L), orc.u8_to_f32(R)
    C = orc.bt_cost(Lf, Rf, 16)
    for sem in (0, 1, 2):
        for table in (0, 1):
            a = orc.sgm(C, Lf, 10, 120, semantics=sem, table=table, threads=1)
            b = orc.sgm(C, Lf, 10, 120, semantics=sem, table=table, threads=4)
            np.testing.assert_array_equal(a[2], b[2])
            np.testing.assert_array_equal(a[0], b[0])


def test_lr_check_small(orc):
    # S for W=4, D=2 (one row); dR(xr) = argmin_d S(xr+d, d)
    S = np.array([[0, 5], [3, 1], [2, 2], [9, 0]], np.float32).reshape(1, 4, 2)
    dL = np.array([[0, 1, 0, 1]], np.uint16)
    dl, dr = orc.lr_check(S, dL, thr=0)
    # dR: xr0 -> min(S(0,0)=0, S(1,1)=1) -> 0; xr1 -> min(3, S(2,1)=2) -> 1;
    #     xr2 -> min(2, S(3,1)=0) -> 1; xr3 -> only d=0 -> 0
    np.testing.assert_array_equal(dr[0], [0, 1, 1, 0])
    # x0: dL 0, dR(0)=0 ok; x1: dL 1 -> dR(0)=0 differs; x2: dL 0, dR(2)=1
    # differs; x3: dL 1 -> dR(2)=1 ok
    np.testing.assert_array_equal(dl[0], [0, 0xFFFF, 0xFFFF, 1])


def test_soft_sgm_gradcheck_fp64(orc):
    rng = np.random.default_rng(7)
    C = rng.uniform(0, 10, size=(4, 5, 3))
    g = rng.normal(size=(4, 5))
    dC, d1, d2 = orc.soft_sgm_bwd(C, 1.3, 4.1, g, tau=0.7)
    eps = 1e-6

    def f(Cx, p1=1.3, p2=4.1):
        _, dh = orc.soft_sgm_fwd(Cx, p1, p2, tau=0.7)
        return float((dh * g).sum())

    for idx in [(0, 0, 0), (1, 2, 1), (3, 4, 2), (2, 3, 0)]:
        Cp, Cm = C.copy(), C.copy()
        Cp[idx] += eps
        Cm[idx] -= eps
        assert dC[idx] == pytest.approx((f(Cp) - f(Cm)) / (2 * eps), rel=1e-5, abs=1e-8)
    assert d1 == pytest.approx((f(C, 1.3 + eps) - f(C, 1.3 - eps)) / (2 * eps), rel=1e-5, abs=1e-8)
    assert d2 == pytest.approx((f(C, p2=4.1 + eps) - f(C, p2=4.1 - eps)) / (2 * eps), rel=1e-5,
                               abs=1e-8)


def test_cost_pair_equals_the_equal_size_costs(orc):
    # the different-size entry point reduces to the three cost functions
    rng = np.random.default_rng(12)
    L = rng.random((9, 23), dtype=np.float32)
    R = rng.random((9, 23), dtype=np.float32)
    for layout in (orc.LAYOUT_HWD, orc.LAYOUT_REF_WHD):
        assert np.array_equal(orc.cost_pair(L, R, 6, 0, 0, layout), orc.bt_cost(L, R, 6, layout))
        assert np.array_equal(orc.cost_pair(L, R, 6, 1, 2, layout), orc.ssd_cost(L, R, 6, 2, layout))
        assert np.array_equal(orc.cost_pair(L, R, 6, 2, 1, layout), orc.ncc_cost(L, R, 6, 1, layout), equal_nan=True)
    # a wider right image: the DSI is the left's width and the right taps
    # read past it instead of clamping
    R2 = np.concatenate([R, rng.random((9, 4), dtype=np.float32)], axis=1)
    a = orc.cost_pair(L, R2, 6, 1, 2)
    assert a.shape == (9, 23, 6)
    assert not np.array_equal(a, orc.ssd_cost(L, R, 6, 2))
    assert np.array_equal(a[:, :20], orc.ssd_cost(L, R, 6, 2)[:, :20])
