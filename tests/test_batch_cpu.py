"""Host side of the batched form, no GPU: the seeded ensemble of independent
rising-bubble cases, and argument checks of ``fugu_batch_create`` that fail
before any device work."""
import ctypes as C

import numpy as np

from coupled_codefort_2d_b200 import cases


def test_ensemble_is_seeded_and_in_range():
    a = cases.bubble_ensemble(256)
    b = cases.bubble_ensemble(256)
    assert a == b
    assert len(a) == 256
    sizes = {(s["grid"].nx, s["grid"].ny) for s in a}
    assert sizes == set(cases.ENSEMBLE_GRIDS)
    for s in a:
        g = s["grid"]
        assert (g.Lx, g.Ly) == (1.0, 2.0) and g.dx == g.dy
        assert 0.15 <= s["radius"] <= 0.3 and 0.4 <= s["xc"] <= 0.6 and s["yc"] == 0.5
        assert 10.0 <= s["rho1"] / s["rho2"] <= 1000.0 and s["rho1"] == 1000.0
        assert 10.0 <= s["mu1"] / s["mu2"] <= 100.0 and s["mu1"] == 10.0
        assert 1.0 <= s["sigma"] <= 50.0 and s["gy"] == -0.98
    # the first cases of a larger ensemble are the same cases (one draw
    # sequence per case, in case order)
    assert cases.bubble_ensemble(8) == a[:8]


def test_ensemble_mean_size_matches_the_grid_mix():
    a = cases.bubble_ensemble(256)
    mean = np.mean([s["grid"].ncells for s in a])
    assert 40_000 < mean < 85_000  # the mix's expectation is 61,440 cells


def test_batch_create_rejects_bad_arguments():
    from coupled_codefort_2d_b200 import _lib
    from coupled_codefort_2d_b200.batch import ensemble_params
    from coupled_codefort_2d_b200.context import make_params

    L = _lib.lib()
    spec = cases.bubble_ensemble(1)[0]
    p = make_params(spec["grid"], ensemble_params(spec))
    arr = (_lib.FuguParams * 1)(p)
    h = C.c_void_p()
    assert L.fugu_batch_create(arr, 0, 0, None, C.byref(h)) == -1
    bad = _lib.FuguBatchOpts(0, 17, 0)  # a cluster holds at most 16 CTAs
    assert L.fugu_batch_create(arr, 1, 0, C.byref(bad), C.byref(h)) == -1
    arr[0].nx = 2
    assert L.fugu_batch_create(arr, 1, 0, None, C.byref(h)) == -1
    assert not h.value
    assert L.fugu_batch_size(None) == 0
