"""Initial colour fields of the benchmark configurations (host side): the
droplet's area fractions by sub-sampling (config C2 asks for 16 x 16), and the
phase convention of the reference (C = 1 is fluid 1; the droplet is fluid 1
inside, the rising bubble is fluid 2 inside, ``src/main.f90:137-166``)."""
import math

import numpy as np

from coupled_codefort_2d_b200 import cases
from coupled_codefort_2d_b200.layout import Grid, at


def test_droplet_area_fractions_integrate_to_the_disc():
    g = Grid(256, 256)
    c = cases.circle_fraction(g, 0.5, 0.5, 0.25, inside=1.0, ns=16)
    inner = at(c, "cell", slice(1, g.nx), slice(1, g.ny))
    area = float(inner.sum()) * g.dx * g.dy
    assert abs(area - math.pi * 0.25 ** 2) < 2e-5  # sub-sampling error, far below one cell (1.5e-5)
    assert inner.min() == 0.0 and inner.max() == 1.0
    # cut cells lie along the circle: about its length over h of them
    cut = int(np.count_nonzero((inner > 0.0) & (inner < 1.0)))
    assert 1.0 * 2 * math.pi * 0.25 / g.dx < cut < 1.6 * 2 * math.pi * 0.25 / g.dx
    assert inner[128, 128] == 1.0 and inner[0, 0] == 0.0  # fluid 1 inside


def test_bubble_is_fluid_two_inside():
    g = Grid(32, 64, 1.0, 2.0)
    c = cases.initial_colour(g, "rising_bubble")
    inner = at(c, "cell", slice(1, g.nx), slice(1, g.ny))
    assert inner[16, 16] == 0.0 and inner[0, 0] == 1.0  # centre (0.5, 0.5) is the bubble
    assert np.all((inner == 0.0) | (inner == 1.0))  # the reference's binary test
