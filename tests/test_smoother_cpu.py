"""The PCD's red-black SOR velocity smoother (extension, ``pcd_smoother = 1``)
in the CPU oracle, pinned against a plain-Python restatement of the sweep.

The reference smooths the velocity blocks of its PCD preconditioner by damped
Jacobi (``src/mod_subsolvers.f90:252-372``).  The extension keeps that
formula (5-point viscous stencil plus rho/dt and the Darcy penalty on the
diagonal, wall faces set to the right-hand side) but updates in place, first
the faces with (i + j) even and then the odd ones, with over-relaxation
omega, refreshing the periodic halo before each colour.  The GPU kernels are
checked bit for bit against this oracle in ``test_gpu_routines.py``.
"""
import numpy as np
import pytest

from conftest import colour, rfield, two_phase_params
from coupled_codefort_2d_b200.layout import Grid, at

GRIDS = {"walls_9x7": Grid(9, 7, 1.0, 0.8), "px_8x6": Grid(8, 6, periodic_x=True),
         "py_7x8": Grid(7, 8, periodic_y=True)}


def _rbsor_u(o, g, u, rhs, pr, dt, sweeps, om):
    """red-black SOR on the u block, element by element"""
    kap, zeta, eta, rho = pr["kappa"], pr["zeta"], pr["eta"], pr["rho_u"]
    ix2, iy2 = 1.0 / (g.dx * g.dx), 1.0 / (g.dy * g.dy)
    imax = g.nx if g.periodic_x else g.nx - 1
    for _ in range(sweeps):
        for col in (0, 1):
            o.halo("u", u)
            for j in range(1, g.ny + 1):
                for i in range(1, imax + 1):
                    if (i + j) & 1 != col:
                        continue
                    cE = at(kap, "cell", i + 1, j) * ix2
                    cW = at(kap, "cell", i, j) * ix2
                    cN = (at(zeta, "vert", i, j) - at(eta, "vert", i, j)) * iy2
                    cS = (at(zeta, "vert", i, j - 1) - at(eta, "vert", i, j - 1)) * iy2
                    diag = (at(rho, "u", i, j) / dt) + cE + cW + cN + cS
                    off = (cE * at(u, "u", i + 1, j) + cW * at(u, "u", i - 1, j) + cN * at(u, "u", i, j + 1)
                           + cS * at(u, "u", i, j - 1))
                    if diag > 1.0e-15:
                        u[i + 2, j + 1] = (1.0 - om) * at(u, "u", i, j) + om * ((at(rhs, "u", i, j) + off) / diag)
                if not g.periodic_x:
                    for i in (0, g.nx):
                        if (i + j) & 1 == col:
                            u[i + 2, j + 1] = at(rhs, "u", i, j)


def _rbsor_v(o, g, v, rhs, pr, dt, sweeps, om):
    """red-black SOR on the v block, element by element"""
    kap, zeta, eta, rho = pr["kappa"], pr["zeta"], pr["eta"], pr["rho_v"]
    ix2, iy2 = 1.0 / (g.dx * g.dx), 1.0 / (g.dy * g.dy)
    jmax = g.ny if g.periodic_y else g.ny - 1
    for _ in range(sweeps):
        for col in (0, 1):
            o.halo("v", v)
            for j in range(1, jmax + 1):
                for i in range(1, g.nx + 1):
                    if (i + j) & 1 != col:
                        continue
                    cE = (at(zeta, "vert", i, j) - at(eta, "vert", i, j)) * ix2
                    cW = (at(zeta, "vert", i - 1, j) - at(eta, "vert", i - 1, j)) * ix2
                    cN = at(kap, "cell", i, j + 1) * iy2
                    cS = at(kap, "cell", i, j) * iy2
                    diag = (at(rho, "v", i, j) / dt) + cE + cW + cN + cS
                    off = (cE * at(v, "v", i + 1, j) + cW * at(v, "v", i - 1, j) + cN * at(v, "v", i, j + 1)
                           + cS * at(v, "v", i, j - 1))
                    if diag > 1.0e-15:
                        v[i + 1, j + 2] = (1.0 - om) * at(v, "v", i, j) + om * ((at(rhs, "v", i, j) + off) / diag)
            if not g.periodic_y:
                for i in range(1, g.nx + 1):
                    for j in (0, g.ny):
                        if (i + j) & 1 == col:
                            v[i + 1, j + 2] = at(rhs, "v", i, j)


def _setup(oracle_mod, g, smoother, om=1.5):
    rng = np.random.default_rng(21)
    prm = two_phase_params(pcd_smoother=smoother, pcd_sor_omega=om)
    o = oracle_mod.Oracle(g, prm)
    pr = o.properties(colour(rng, g))
    return rng, o, pr


@pytest.mark.parametrize("gname", list(GRIDS))
def test_oracle_rbsor_matches_restatement(oracle_mod, gname):
    g = GRIDS[gname]
    rng, o, pr = _setup(oracle_mod, g, 1)
    u0, rhs = rfield(rng, g, "u"), rfield(rng, g, "u")
    a, b = u0.copy(order="F"), u0.copy(order="F")
    o.helmholtz_u(a, rhs, pr, 2e-3, 3)
    _rbsor_u(o, g, b, rhs, pr, 2e-3, 3, 1.5)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("gname", list(GRIDS))
def test_oracle_rbsor_v_matches_restatement(oracle_mod, gname):
    g = GRIDS[gname]
    rng, o, pr = _setup(oracle_mod, g, 1)
    v0, rhs = rfield(rng, g, "v"), rfield(rng, g, "v")
    a, b = v0.copy(order="F"), v0.copy(order="F")
    o.helmholtz_v(a, rhs, pr, 2e-3, 3)
    _rbsor_v(o, g, b, rhs, pr, 2e-3, 3, 1.5)
    np.testing.assert_array_equal(a, b)


def _residual_u(o, g, u, rhs, pr, dt):
    """max |rhs - A u| over the owned u faces"""
    w = u.copy(order="F")
    o.halo("u", w)
    kap, zeta, eta, rho = pr["kappa"], pr["zeta"], pr["eta"], pr["rho_u"]
    ix2, iy2 = 1.0 / (g.dx * g.dx), 1.0 / (g.dy * g.dy)
    imax = g.nx if g.periodic_x else g.nx - 1
    r = 0.0
    for j in range(1, g.ny + 1):
        for i in range(1, imax + 1):
            cE = at(kap, "cell", i + 1, j) * ix2
            cW = at(kap, "cell", i, j) * ix2
            cN = (at(zeta, "vert", i, j) - at(eta, "vert", i, j)) * iy2
            cS = (at(zeta, "vert", i, j - 1) - at(eta, "vert", i, j - 1)) * iy2
            diag = at(rho, "u", i, j) / dt + cE + cW + cN + cS
            au = diag * at(w, "u", i, j) - (cE * at(w, "u", i + 1, j) + cW * at(w, "u", i - 1, j)
                                            + cN * at(w, "u", i, j + 1) + cS * at(w, "u", i, j - 1))
            r = max(r, abs(at(rhs, "u", i, j) - au))
    return r


def test_rbsor_reduces_the_residual_faster_than_jacobi(oracle_mod):
    """On a viscous-dominated block (large dt), 6 red-black SOR sweeps leave a
    smaller residual than 6 damped-Jacobi sweeps, which is why the batched
    rising-bubble cases need fewer Arnoldi steps with it."""
    g = Grid(24, 20)
    res = {}
    for sm in (0, 1):
        rng, o, pr = _setup(oracle_mod, g, sm)
        rhs = rfield(rng, g, "u")
        u = g.zeros("u")
        o.helmholtz_u(u, rhs, pr, 1.0, 6)
        res[sm] = _residual_u(o, g, u, rhs, pr, 1.0)
    assert res[1] < 0.5 * res[0], res
