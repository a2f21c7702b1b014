"""Case initialisers and diagnostics of the FUGU-2D driver and tests.

Colour-function initialisers follow ``src/main.f90:135-183`` (binary ``r <= R``
test evaluated at every cell centre, ghosts included, then a halo exchange).
``circle_fraction`` is the extension the droplet benchmark asks for: exact
area fractions by ``ns x ns`` sub-sampling.  ``C = 1`` is fluid 1
(``mod_viscosity.f90:68``).

Diagnostics restate the reference tests' formulas (file:line in each
docstring).
"""
from __future__ import annotations

import numpy as np

from .layout import Grid, at


def _centres(g: Grid):
    # cell centres of the padded cell array, i = -1..nx+2 (i_start = 1)
    i = np.arange(-1, g.nx + 3, dtype=np.float64)
    j = np.arange(-1, g.ny + 3, dtype=np.float64)
    xc = (i - 0.5) * g.dx
    yc = (j - 0.5) * g.dy
    return np.meshgrid(xc, yc, indexing="ij")


def periodic_wrap_cell(g: Grid, c: np.ndarray) -> np.ndarray:
    """Single-rank ``mpi_exchange_halos_scalar`` (``mod_mpi.f90:113-153``)."""
    nx, ny = g.nx, g.ny
    if g.periodic_x:
        c[0:2, :] = c[nx:nx + 2, :].copy()
        c[nx + 2:nx + 4, :] = c[2:4, :].copy()
    if g.periodic_y:
        c[:, 0:2] = c[:, ny:ny + 2].copy()
        c[:, ny + 2:ny + 4] = c[:, 2:4].copy()
    return c


def binary_circle(g: Grid, xc: float, yc: float, radius: float, inside: float) -> np.ndarray:
    """``C = inside`` where the cell centre lies within ``radius``
    (``main.f90:137-166``)."""
    X, Y = _centres(g)
    r = np.sqrt((X - xc) ** 2 + (Y - yc) ** 2)
    c = np.where(r <= radius, inside, 1.0 - inside).astype(np.float64)
    return periodic_wrap_cell(g, np.asfortranarray(c))


def circle_fraction(g: Grid, xc: float, yc: float, radius: float, inside: float,
                    ns: int = 16) -> np.ndarray:
    """Area fraction of a circle in each cell by ``ns x ns`` sub-sampling
    (extension; the reference uses the binary test).  ``inside`` is the C
    value of the disc."""
    X, Y = _centres(g)
    off = (np.arange(ns, dtype=np.float64) + 0.5) / ns - 0.5
    frac = np.zeros_like(X)
    for a in off:
        for b in off:
            frac += ((X + a * g.dx - xc) ** 2 + (Y + b * g.dy - yc) ** 2) <= radius * radius
    frac /= ns * ns
    c = inside * frac + (1.0 - inside) * (1.0 - frac)
    return periodic_wrap_cell(g, np.asfortranarray(c))


def poiseuille_layers(g: Grid) -> np.ndarray:
    """``C = 1`` below ``y = Ly/2`` (``main.f90:167-178``)."""
    _, Y = _centres(g)
    c = np.where(Y <= 0.5 * g.Ly, 1.0, 0.0)
    return periodic_wrap_cell(g, np.asfortranarray(c))


def initial_colour(g: Grid, case_type: str, drop_rad: float = 0.25) -> np.ndarray:
    """Colour function of the driver's named cases (``main.f90:135-183``)."""
    if case_type == "rising_bubble":
        return binary_circle(g, 0.5 * g.Lx, 0.5, drop_rad, inside=0.0)
    if case_type == "laplace":
        return binary_circle(g, 0.5 * g.Lx, 0.5 * g.Ly, drop_rad, inside=1.0)
    if case_type == "poiseuille":
        return poiseuille_layers(g)
    return g.full("cell", 1.0)


# ---------------------------------------------------------------- diagnostics
def cell_centres_interior(g: Grid):
    x = (np.arange(1, g.nx + 1) - 0.5) * g.dx
    y = (np.arange(1, g.ny + 1) - 0.5) * g.dy
    return np.meshgrid(x, y, indexing="ij")


def bubble_volume(g: Grid, c: np.ndarray) -> float:
    """Volume of fluid 2 (``test_rising_bubble.f90:137-147``)."""
    ci = at(c, "cell", slice(1, g.nx), slice(1, g.ny))
    return float(np.sum((1.0 - ci) * g.dx * g.dy))


def fluid1_volume(g: Grid, c: np.ndarray) -> float:
    """Volume of fluid 1 (``test_laplace_coupled.f90:517-524``)."""
    ci = at(c, "cell", slice(1, g.nx), slice(1, g.ny))
    return float(np.sum(ci * g.dx * g.dy))


def bubble_centroid_velocity(g: Grid, c: np.ndarray, v: np.ndarray):
    """Centroid height and rise velocity of fluid 2
    (``test_rising_bubble.f90:134-155``)."""
    ci = at(c, "cell", slice(1, g.nx), slice(1, g.ny))
    _, Y = cell_centres_interior(g)
    vb = 1.0 - ci
    vcell = 0.5 * (at(v, "v", slice(1, g.nx), slice(0, g.ny - 1)) + at(v, "v", slice(1, g.nx), slice(1, g.ny)))
    vol = np.sum(vb) * g.dx * g.dy
    ycm = np.sum(vb * Y) * g.dx * g.dy / max(vol, 1e-14)
    vr = np.sum(vb * vcell) * g.dx * g.dy / max(vol, 1e-14)
    return float(ycm), float(vr)


def circularity(g: Grid, c: np.ndarray, level: float = 0.5) -> float:
    """Degree of circularity of the fluid-2 region: perimeter of the
    area-equivalent circle over the interface perimeter, the perimeter being
    the sum of |grad C| dA (a smooth-indicator estimate)."""
    ci = at(c, "cell", slice(1, g.nx), slice(1, g.ny))
    area = np.sum(1.0 - ci) * g.dx * g.dy
    gx = np.zeros_like(ci)
    gy = np.zeros_like(ci)
    gx[1:-1, :] = (ci[2:, :] - ci[:-2, :]) / (2 * g.dx)
    gy[:, 1:-1] = (ci[:, 2:] - ci[:, :-2]) / (2 * g.dy)
    perim = np.sum(np.sqrt(gx * gx + gy * gy)) * g.dx * g.dy
    return float(2.0 * np.sqrt(np.pi * area) / max(perim, 1e-300))


def laplace_jump(g: Grid, p: np.ndarray, radius: float, xc: float = 0.5, yc: float = 0.5) -> float:
    """Mean pressure inside r < 0.7R minus outside r > 1.3R
    (``test_laplace_coupled.f90:527-556``)."""
    X, Y = cell_centres_interior(g)
    r = np.sqrt((X - xc) ** 2 + (Y - yc) ** 2)
    pi_ = at(p, "cell", slice(1, g.nx), slice(1, g.ny))
    pin = pi_[r < 0.7 * radius]
    pout = pi_[r > 1.3 * radius]
    return float(pin.sum() / max(pin.size, 1) - pout.sum() / max(pout.size, 1))


def max_divergence(g: Grid, u: np.ndarray, v: np.ndarray) -> float:
    """max |div u| over cells (``op_divergence``, ``mod_operators.f90:34-53``)."""
    du = (at(u, "u", slice(1, g.nx), slice(1, g.ny)) - at(u, "u", slice(0, g.nx - 1), slice(1, g.ny))) / g.dx
    dv = (at(v, "v", slice(1, g.nx), slice(1, g.ny)) - at(v, "v", slice(1, g.nx), slice(0, g.ny - 1))) / g.dy
    return float(np.max(np.abs(du + dv)))


# ------------------------------------------------------- batched ensemble
ENSEMBLE_GRIDS = ((64, 128), (128, 256), (192, 384), (256, 512))
ENSEMBLE_SEED = 20261203


def bubble_ensemble(ncases: int, seed: int = ENSEMBLE_SEED, grids=ENSEMBLE_GRIDS):
    """Independent two-phase rising-bubble cases in a 1 x 2 box.

    One draw sequence per case, in case order, from
    ``numpy.random.default_rng(seed)``: grid uniform over ``grids``; radius
    ``U[0.15, 0.3] * Lx``; centre ``x = U[0.4, 0.6] * Lx``, ``y = 0.5``;
    ``rho_out / rho_in`` log-uniform in [10, 1000] with ``rho_out = 1000``;
    ``mu_out / mu_in`` log-uniform in [10, 100] with ``mu_out = 10``;
    ``sigma = U[1, 50]``; ``g = 0.98`` downwards.  The bubble is fluid 2
    (``C = 0``, the reference's ``rising_bubble`` colour, ``main.f90:137-150``),
    top and bottom walls are no-slip and the side walls free-slip.  Returns
    dicts with the grid, the physics and the bubble geometry; the solver
    settings are the caller's.
    """
    rng = np.random.default_rng(seed)
    out = []
    for k in range(ncases):
        nx, ny = grids[int(rng.integers(len(grids)))]
        radius = float(rng.uniform(0.15, 0.3))
        xc = float(rng.uniform(0.4, 0.6))
        rho_ratio = float(np.exp(rng.uniform(np.log(10.0), np.log(1000.0))))
        mu_ratio = float(np.exp(rng.uniform(np.log(10.0), np.log(100.0))))
        sigma = float(rng.uniform(1.0, 50.0))
        out.append({
            "case": k, "grid": Grid(nx, ny, 1.0, 2.0), "radius": radius, "xc": xc, "yc": 0.5,
            "rho1": 1000.0, "rho2": 1000.0 / rho_ratio, "mu1": 10.0, "mu2": 10.0 / mu_ratio,
            "sigma": sigma, "gx": 0.0, "gy": -0.98,
        })
    return out
