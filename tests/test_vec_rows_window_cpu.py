"""The load rules of the vectorised row kernels (``k_jacobi_vec``,
``k_pcd_schur_vec``, ``k_pcd_zwork_vec``, ``k_pcd_cross_vec`` in
``csrc/kernels.cuh``), restated in Python and checked on the CPU.

A thread of those kernels takes W = 16 / sizeof(T) elements of one box row
(W = 4 in FP32, 2 in FP64), loads what the element functions need into a
window of registers -- rows j - 1, j, j + 1 of the columns i0 - 1 .. i0 + W,
each part only under the kernel's own conditions -- and evaluates the same
element functions through the window.  Here every slot the kernel does not
load holds NaN, every load is checked to stay inside the padded box, and
each element's value through the window must equal its value from the whole
arrays: a read of a slot the kernel never filled would show up as NaN.  The
formulas are those of ``jacobi_u_vals`` / ``jacobi_v_vals``
(``src/mod_subsolvers.f90:284-306, 346-369``) and the PCD steps
(``src/mod_pcd_precond.f90:54-98``).  The GPU kernels themselves are checked
against the oracle bit for bit in ``tests/test_gpu_vec_rows.py``.
"""
import math

import numpy as np
import pytest

from test_rbsor_tiling_cpu import Box

NAN = float("nan")


class PBox(Box):
    def __init__(self, nx, ny, px=False, py=False):
        super().__init__(nx, ny)
        self.px, self.py = px, py

    @property
    def imax(self):
        return self.nx if self.px else self.nx - 1

    @property
    def jmax(self):
        return self.ny if self.py else self.ny - 1


class Whole:
    """a field of the box read at Fortran (i, j)"""

    def __init__(self, g, a):
        self.g, self.a = g, a

    def __call__(self, i, j):
        return self.a[self.g.at(i, j)]


class Window:
    """the kernel's register window of one field for the segment starting at
    box column ii0 of box row jj; unfilled slots read NaN"""

    def __init__(self, g, a, W, ii0, jj):
        self.g, self.a, self.W, self.ii0, self.jj = g, a, W, ii0, jj
        self.i0, self.j0 = ii0 - 2, jj - 2
        self.v = {}

    def row(self, r, left=False, right=False):
        """slot row r (0: j - 1, 1: j, 2: j + 1): W elements, plus the
        neighbours either side when asked, each load inside the box"""
        g, jrow = self.g, self.jj + r - 1
        assert 0 <= jrow < g.R, ("row outside the box", jrow)
        cols = list(range(self.W))
        if left:
            cols.append(-1)
        if right:
            cols.append(self.W)
        for c in cols:
            ii = self.ii0 + c
            assert 0 <= ii < g.P, ("column outside the box", ii)
            self.v[(r, c)] = self.a[ii + jrow * g.P]
        return self

    def __call__(self, i, j):
        return self.v.get((j - self.j0 + 1, i - self.i0), NAN)


def jac_u(g, i, j, U, K, Z, E, rhs, rho, pen, ix2, iy2, dt, om):
    val = U(i, j)
    if 1 <= j <= g.ny:
        if 1 <= i <= g.imax:
            cE, cW = K(i + 1, j) * ix2, K(i, j) * ix2
            cN, cS = (Z(i, j) - E(i, j)) * iy2, (Z(i, j - 1) - E(i, j - 1)) * iy2
            diag = rho / dt + cE + cW + cN + cS + pen
            off = cS * U(i, j - 1) + (cN * U(i, j + 1) + (cW * U(i - 1, j) + cE * U(i + 1, j)))
            if diag > 1e-15:
                val = (1 - om) * U(i, j) + om * ((rhs + off) / diag)
        elif not g.px and i in (0, g.nx):
            val = rhs
    return val


def jac_v(g, i, j, U, K, Z, E, rhs, rho, pen, ix2, iy2, dt, om):
    val = U(i, j)
    if 1 <= i <= g.nx:
        if 1 <= j <= g.jmax:
            cE, cW = (Z(i, j) - E(i, j)) * ix2, (Z(i - 1, j) - E(i - 1, j)) * ix2
            cN, cS = K(i, j + 1) * iy2, K(i, j) * iy2
            diag = rho / dt + cE + cW + cN + cS + pen
            off = cS * U(i, j - 1) + (cN * U(i, j + 1) + (cW * U(i - 1, j) + cE * U(i + 1, j)))
            if diag > 1e-15:
                val = (1 - om) * U(i, j) + om * ((rhs + off) / diag)
        elif not g.py and j in (0, g.ny):
            val = rhs
    return val


def schur(g, i, j, F, A, B, K, Z, inv_dt, visc, idx, idy):
    if 1 <= i <= g.nx and 1 <= j <= g.ny:
        uavg, vavg = 0.5 * (A(i, j) + A(i - 1, j)), 0.5 * (B(i, j) + B(i, j - 1))
        conv = uavg * (F(i + 1, j) - F(i - 1, j)) * (0.5 * idx) + vavg * (F(i, j + 1) - F(i, j - 1)) * (0.5 * idy)
        r = -(inv_dt * F(i, j) + conv)
        if visc:
            r = r - ((visc * 0.5) * K(i, j)) * Z(i, j)
        return r
    return 0.0


def zwork(g, i, j, zu, zv, R, idx, idy):
    a = b = 0.0
    if 1 <= j <= g.ny:
        if 1 <= i <= g.nx - 1:
            a = zu - (R(i + 1, j) - R(i, j)) * idx
        elif i in (0, g.nx):
            a = zu
    if 1 <= i <= g.nx:
        if 1 <= j <= g.ny - 1:
            b = zv - (R(i, j + 1) - R(i, j)) * idy
        elif j in (0, g.ny):
            b = zv
    return a, b


def cross(g, i, j, E, V, z, idx, idy):
    if 1 <= j <= g.ny and 1 <= i <= g.nx - 1:
        return z - (-idy * (E(i, j) * (V(i + 1, j) - V(i, j)) * idx - E(i, j - 1) * (V(i + 1, j - 1) - V(i, j - 1)) * idx))
    return z


BOXES = {"walls_13x9": (13, 9, False, False), "px_16x12": (16, 12, True, False), "py_12x16": (12, 16, False, True),
         "pxy_10x14": (10, 14, True, True), "walls_61x47": (61, 47, False, False)}


def segments(g, W):
    for jj in range(g.R):
        for ii0 in range(0, g.P, W):
            yield ii0, jj


def same(a, b):
    assert not math.isnan(a), "the window read a slot the kernel does not load"
    assert a == b


@pytest.mark.parametrize("W", [2, 4])
@pytest.mark.parametrize("box", list(BOXES))
def test_jacobi_window(box, W):
    g = PBox(*BOXES[box])
    rng = np.random.default_rng(5)
    f = {k: rng.uniform(0.01, 1.0, g.P * g.R) for k in ("u", "rhs", "rho", "kap", "zeta", "eta", "pen")}
    f["eta"] *= 0.01
    ix2, iy2, dt, om = 90.0, 70.0, 2e-3, 0.8
    whole = {k: Whole(g, a) for k, a in f.items()}
    for comp, fn in ((0, jac_u), (1, jac_v)):
        for ii0, jj in segments(g, W):
            lft, rgt = ii0 > 0, ii0 + W < g.P
            j = jj - 2
            U = Window(g, f["u"], W, ii0, jj).row(1, lft, rgt)
            K, Z, E = (Window(g, f[k], W, ii0, jj) for k in ("kap", "zeta", "eta"))
            if 1 <= j <= (g.ny if comp == 0 else g.jmax):  # the stencil rows
                U.row(0, lft, rgt).row(2, lft, rgt)
                if comp == 0:
                    K.row(1, False, rgt)
                    Z.row(1).row(0)
                    E.row(1).row(0)
                else:
                    K.row(1).row(2)
                    Z.row(1, lft, False)
                    E.row(1, lft, False)
            for e in range(W):
                k = ii0 + e + jj * g.P
                i = ii0 + e - 2
                args = (f["rhs"][k], f["rho"][k], f["pen"][k], ix2, iy2, dt, om)
                same(fn(g, i, j, U, K, Z, E, *args),
                     fn(g, i, j, whole["u"], whole["kap"], whole["zeta"], whole["eta"], *args))


@pytest.mark.parametrize("W", [2, 4])
@pytest.mark.parametrize("box", list(BOXES))
@pytest.mark.parametrize("visc", [0.0, 1.0])
def test_pcd_windows(box, W, visc):
    g = PBox(*BOXES[box])
    rng = np.random.default_rng(6)
    f = {k: rng.uniform(-1.0, 1.0, g.P * g.R) for k in ("phi", "ua", "va", "kap", "zp", "zu", "zv", "rp", "eta", "rv",
                                                         "zuw")}
    w = {k: Whole(g, a) for k, a in f.items()}
    idx, idy, inv_dt = 13.0, 9.0, 500.0
    for ii0, jj in segments(g, W):
        lft, rgt = ii0 > 0, ii0 + W < g.P
        j = jj - 2
        win = {k: Window(g, a, W, ii0, jj) for k, a in f.items()}
        if 1 <= j <= g.ny:  # k_pcd_schur_vec
            win["phi"].row(0).row(1, lft, rgt).row(2)
            win["ua"].row(1, lft, False)
            win["va"].row(1).row(0)
            if visc:
                win["kap"].row(1)
                win["zp"].row(1)
        if 1 <= j <= g.ny:  # k_pcd_zwork_vec
            win["rp"].row(1, False, rgt)
            if j <= g.ny - 1:
                win["rp"].row(2)
        if 1 <= j <= g.ny:  # k_pcd_cross_vec
            win["eta"].row(1).row(0)
            win["rv"].row(1, False, rgt).row(0, False, rgt)
        for e in range(W):
            k = ii0 + e + jj * g.P
            i = ii0 + e - 2
            same(schur(g, i, j, win["phi"], win["ua"], win["va"], win["kap"], win["zp"], inv_dt, visc, idx, idy),
                 schur(g, i, j, w["phi"], w["ua"], w["va"], w["kap"], w["zp"], inv_dt, visc, idx, idy))
            (a0, b0), (a1, b1) = (zwork(g, i, j, f["zu"][k], f["zv"][k], R, idx, idy) for R in (win["rp"], w["rp"]))
            same(a0, a1)
            same(b0, b1)
            if 1 <= j <= g.ny:  # the kernel leaves zuw alone on the other rows
                same(cross(g, i, j, win["eta"], win["rv"], f["zuw"][k], idx, idy),
                     cross(g, i, j, w["eta"], w["rv"], f["zuw"][k], idx, idy))
