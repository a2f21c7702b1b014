"""The tile schedule of the fused red-black SOR sweep (``k_rbsor_sweep`` in
``csrc/kernels.cuh``), restated in Python and checked against the plain
two-colour sweep it replaces.

The fused kernel does a whole sweep (red faces, then black faces) per tile of
RB_TX x RB_TY faces: it stages the tile and a ring of two faces of the input
buffer, forms the coefficients of the tile and a ring of one, updates the red
faces of the tile and of that ring, then the black faces of the tile, and
writes the tile to the OUTPUT buffer.  A face's red neighbours outside the
tile are recomputed from the staged ring, so the result must equal the two
in-place colour passes of the damped-Jacobi formula (``jacobi_u_at`` /
``jacobi_v_at``, ``src/mod_subsolvers.f90:284-306, 346-369``) bit for bit,
whatever the tile order.  Done in place, a tile would read ring values that a
neighbouring tile has already swept: the last test shows that such an order
does change the result, which is why the kernel reads one buffer and writes
the other.  The GPU kernel itself is checked against the oracle's sweep in
``tests/test_gpu_routines.py``.
"""
import os
import re

import numpy as np
import pytest

KERNELS = os.path.join(os.path.dirname(__file__), "..", "coupled_codefort_2d_b200", "csrc", "kernels.cuh")


def _tile_shape():
    src = open(KERNELS).read()
    m = re.search(r"constexpr int RB_TX = (\d+), RB_TY = (\d+);", src)
    assert m, "tile constants not found"
    return int(m.group(1)), int(m.group(2))


TX, TY = _tile_shape()


class Box:
    def __init__(self, nx, ny):
        self.nx, self.ny = nx, ny
        self.P = ((nx + 5 + 15) // 16) * 16
        self.R = ny + 5

    def at(self, i, j):
        return (i + 2) + (j + 2) * self.P


def coefs(comp, g, f, i, j, ix2, iy2, dt):
    """(kind, (cE, cW, cN, cS, diag)): kind 1 owned face, 2 wall face, 0 none"""
    k = g.at(i, j)
    kap, zeta, eta, rho, pen = f["kap"], f["zeta"], f["eta"], f["rho"], f["pen"]
    if comp == 0:
        if not 1 <= j <= g.ny:
            return 0, None
        if 1 <= i <= g.nx - 1:
            e, w = kap[g.at(i + 1, j)] * ix2, kap[k] * ix2
            n, s = (zeta[k] - eta[k]) * iy2, (zeta[g.at(i, j - 1)] - eta[g.at(i, j - 1)]) * iy2
        else:
            return (2, None) if i in (0, g.nx) else (0, None)
    else:
        if not 1 <= i <= g.nx:
            return 0, None
        if 1 <= j <= g.ny - 1:
            e, w = (zeta[k] - eta[k]) * ix2, (zeta[g.at(i - 1, j)] - eta[g.at(i - 1, j)]) * ix2
            n, s = kap[g.at(i, j + 1)] * iy2, kap[k] * iy2
        else:
            return (2, None) if j in (0, g.ny) else (0, None)
    return 1, (e, w, n, s, rho[k] / dt + e + w + n + s + pen[k])


def update(kd, c, rh, uo, uE, uW, uN, uS, om):
    if kd == 2:
        return rh
    e, w, n, s, d = c
    if d > 1e-15:
        return (1 - om) * uo + om * ((rh + (s * uS + (n * uN + (w * uW + e * uE)))) / d)
    return uo


def two_pass(comp, g, u, f, ix2, iy2, dt, om):
    """the two in-place colour passes"""
    u = u.copy()
    for col in (0, 1):
        for jj in range(g.R):
            for ii in range(g.P):
                i, j = ii - 2, jj - 2
                if (i + j) & 1 != col:
                    continue
                kd, c = coefs(comp, g, f, i, j, ix2, iy2, dt)
                if kd == 1:
                    u[g.at(i, j)] = update(kd, c, f["rhs"][g.at(i, j)], u[g.at(i, j)], u[g.at(i + 1, j)],
                                           u[g.at(i - 1, j)], u[g.at(i, j + 1)], u[g.at(i, j - 1)], om)
                elif kd == 2:
                    u[g.at(i, j)] = f["rhs"][g.at(i, j)]
    return u


def tiled(comp, g, uin, f, ix2, iy2, dt, om, uout=None, order=None):
    """the kernel's schedule, one tile after another (in the given order)"""
    SX, SY, CX, CY = TX + 4, TY + 4, TX + 2, TY + 2
    if uout is None:
        uout = np.full_like(uin, np.nan)  # every element of the box must be written
    tiles = [(tx, ty) for ty in range((g.R + TY - 1) // TY) for tx in range((g.P + TX - 1) // TX)]
    for tx, ty in (order(tiles) if order else tiles):
        ii0, jj0 = tx * TX - 2, ty * TY - 2
        su = np.zeros((SY, SX))
        for b in range(SY):
            for a in range(SX):
                ii, jj = ii0 + a, jj0 + b
                if 0 <= ii < g.P and 0 <= jj < g.R:
                    su[b, a] = uin[ii + jj * g.P]
        kind, cc, rh = np.zeros((CY, CX), int), {}, {}
        for b in range(CY):
            for a in range(CX):
                ii, jj = ii0 + 1 + a, jj0 + 1 + b
                if 0 <= ii < g.P and 0 <= jj < g.R:
                    kd, c = coefs(comp, g, f, ii - 2, jj - 2, ix2, iy2, dt)
                    kind[b, a], cc[b, a] = kd, c
                    if kd:
                        rh[b, a] = f["rhs"][ii + jj * g.P]
        for col in (0, 1):  # red on the tile and its ring, black on the tile
            lo, cx, cy = (0, CX, CY) if col == 0 else (1, TX, TY)
            for q in range(cx * cy):
                a, b = lo + q % cx, lo + q // cx
                i, j = ii0 + a - 1, jj0 + b - 1
                if not kind[b, a] or (i + j) & 1 != col:
                    continue
                ua, ub = a + 1, b + 1
                su[ub, ua] = update(kind[b, a], cc[b, a], rh[b, a], su[ub, ua], su[ub, ua + 1], su[ub, ua - 1],
                                    su[ub + 1, ua], su[ub - 1, ua], om)
        for q in range(TX * TY):
            a, b = 1 + q % TX, 1 + q // TX
            ii, jj = ii0 + 1 + a, jj0 + 1 + b
            if ii < g.P and jj < g.R:
                uout[ii + jj * g.P] = su[b + 1, a + 1]
    return uout


def fields(g, seed):
    rng = np.random.default_rng(seed)
    n = g.P * g.R
    f = {k: rng.uniform(0.5, 2.0, n) for k in ("kap", "zeta", "rho", "rhs", "pen")}
    f["eta"] = rng.uniform(0.0, 0.4, n)
    return f, rng.uniform(-1.0, 1.0, n)


@pytest.mark.parametrize("nx,ny", [(13, 9), (40, 21), (33, 35)])
@pytest.mark.parametrize("comp", [0, 1])
def test_tiled_sweep_equals_two_colour_passes(nx, ny, comp):
    g = Box(nx, ny)
    f, u0 = fields(g, 7 * nx + ny + comp)
    ref = two_pass(comp, g, u0, f, 3.0, 5.0, 0.1, 1.5)
    out = tiled(comp, g, u0, f, 3.0, 5.0, 0.1, 1.5)
    assert not np.isnan(out).any()
    assert np.array_equal(out, ref)
    assert np.sum(ref != u0) > nx * ny // 2  # the sweep did change the box


def test_tile_order_does_not_matter_with_two_buffers():
    g = Box(40, 35)
    f, u0 = fields(g, 3)
    fwd = tiled(0, g, u0, f, 3.0, 5.0, 0.1, 1.5)
    rev = tiled(0, g, u0, f, 3.0, 5.0, 0.1, 1.5, order=lambda t: t[::-1])
    assert np.array_equal(fwd, rev)


def test_in_place_tiles_read_swept_neighbours():
    """one buffer for input and output: a tile then stages ring values that an
    earlier tile has already swept, and the result moves off the two passes"""
    g = Box(40, 35)
    f, u0 = fields(g, 3)
    ref = two_pass(0, g, u0, f, 3.0, 5.0, 0.1, 1.5)
    buf = u0.copy()
    tiled(0, g, buf, f, 3.0, 5.0, 0.1, 1.5, uout=buf)
    assert not np.array_equal(buf, ref)
