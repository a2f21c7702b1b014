"""The tile schedule of the multi-sweep damped-Jacobi kernel
(``k_jacobi_multi`` in ``csrc/kernels.cuh``), restated in Python and checked
against the one-sweep-per-launch Jacobi it replaces.

The kernel does up to JM_K sweeps of one velocity component per tile of
JM_TX x JM_TY faces: it stages the tile and a ring of JM_K faces of the input,
forms the coefficients of the tile and a ring of JM_K - 1 once, and sweep s of
nsw updates the tile and a ring of nsw - s faces from the previous sweep's
values; faces keep the damped-Jacobi formula of ``jacobi_u_vals`` /
``jacobi_v_vals`` (``src/mod_subsolvers.f90:284-306, 346-369``), wall faces
take the right-hand side, other elements keep their value.  The result must
equal nsw separate whole-box sweeps bit for bit, whatever nsw <= JM_K, and
leave no element of the box unwritten.  The GPU kernel itself is checked
against the oracle in ``tests/test_gpu_routines.py``.
"""
import os
import re

import numpy as np
import pytest

from test_rbsor_tiling_cpu import Box, coefs, fields

KERNELS = os.path.join(os.path.dirname(__file__), "..", "coupled_codefort_2d_b200", "csrc", "kernels.cuh")


def _shape():
    src = open(KERNELS).read()
    m = re.search(r"constexpr int JM_TX = (\d+), JM_TY = (\d+), JM_K = (\d+)", src)
    assert m, "tile constants not found"
    return int(m.group(1)), int(m.group(2)), int(m.group(3))


TX, TY, K = _shape()


def jacobi_value(kd, c, rh, uo, uE, uW, uN, uS, om):
    if kd == 2:
        return rh
    if kd == 0:
        return uo
    e, w, n, s, d = c
    if d > 1e-15:
        return (1 - om) * uo + om * ((rh + (s * uS + (n * uN + (w * uW + e * uE)))) / d)
    return uo


def whole_box_sweeps(comp, g, u, f, ix2, iy2, dt, om, nsw):
    for _ in range(nsw):
        new = u.copy()
        for jj in range(g.R):
            for ii in range(g.P):
                i, j = ii - 2, jj - 2
                kd, c = coefs(comp, g, f, i, j, ix2, iy2, dt)
                k = g.at(i, j)
                if kd == 1:
                    new[k] = jacobi_value(kd, c, f["rhs"][k], u[k], u[g.at(i + 1, j)], u[g.at(i - 1, j)],
                                          u[g.at(i, j + 1)], u[g.at(i, j - 1)], om)
                elif kd == 2:
                    new[k] = f["rhs"][k]
        u = new
    return u


def tiled(comp, g, uin, f, ix2, iy2, dt, om, nsw):
    SX, SY = TX + 16, TY + 2 * K
    CX, CY = TX + 2 * (K - 1), TY + 2 * (K - 1)
    uout = np.full_like(uin, np.nan)
    for ty in range((g.R + TY - 1) // TY):
        for tx in range((g.P + TX - 1) // TX):
            ii0, jj0 = tx * TX, ty * TY
            sx0, sy0, cx0, cy0 = ii0 - 8, jj0 - K, ii0 - (K - 1), jj0 - (K - 1)
            u = [np.zeros((SY, SX)), np.zeros((SY, SX))]
            for b in range(SY):
                for a in range(SX):
                    ii, jj = sx0 + a, sy0 + b
                    if 0 <= ii < g.P and 0 <= jj < g.R:
                        u[0][b, a] = uin[ii + jj * g.P]
            kind, cc, rh = np.zeros((CY, CX), int), {}, {}
            for b in range(CY):
                for a in range(CX):
                    ii, jj = cx0 + a, cy0 + b
                    if 0 <= ii < g.P and 0 <= jj < g.R:
                        kd, c = coefs(comp, g, f, ii - 2, jj - 2, ix2, iy2, dt)
                        kind[b, a], cc[b, a] = kd, c
                        if kd:
                            rh[b, a] = f["rhs"][ii + jj * g.P]
            cur = 0
            for sweep in range(1, nsw + 1):
                ring = nsw - sweep
                for jj in range(jj0 - ring, jj0 + TY + ring):
                    for ii in range(ii0 - ring, ii0 + TX + ring):
                        a, b, ua, ub = ii - cx0, jj - cy0, ii - sx0, jj - sy0
                        src = u[cur]
                        u[cur ^ 1][ub, ua] = jacobi_value(kind[b, a], cc.get((b, a)), rh.get((b, a)), src[ub, ua],
                                                          src[ub, ua + 1], src[ub, ua - 1], src[ub + 1, ua],
                                                          src[ub - 1, ua], om)
                cur ^= 1
            for jj in range(jj0, jj0 + TY):
                for ii in range(ii0, ii0 + TX):
                    if ii < g.P and jj < g.R:
                        uout[ii + jj * g.P] = u[cur][jj - sy0, ii - sx0]
    return uout


@pytest.mark.parametrize("nx,ny,comp,nsw", [(13, 9, 0, K), (40, 21, 1, K), (33, 20, 0, 3), (20, 33, 1, 1)])
def test_tiled_sweeps_equal_whole_box_sweeps(nx, ny, comp, nsw):
    g = Box(nx, ny)
    f, u0 = fields(g, 11 * nx + ny + comp)
    ref = whole_box_sweeps(comp, g, u0, f, 3.0, 5.0, 0.1, 0.8, nsw)
    out = tiled(comp, g, u0, f, 3.0, 5.0, 0.1, 0.8, nsw)
    assert not np.isnan(out).any()
    assert np.array_equal(out, ref)
    assert np.sum(ref != u0) > nx * ny // 2
