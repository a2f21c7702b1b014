"""The allocation-free Poisson entry, fugu_solve_poisson_pressure_noalloc,
against the context entry fugu_solve_poisson_pressure on the same inputs.

The allocation-free entry runs the grid-wide PCG kernel on a static device
array; the context entry picks its own PCG kernel.  Both accumulate the PCG
scalars error-free, so the test tolerance (1e-12 relative on phi and the
residual, the same iteration count) is far above what the two can differ by.
Two calls in a row (two different cases) check that nothing of one call
leaks into the next.  This file is collected last on purpose: the entry must
work both in a fresh process and after every other GPU test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import GRIDS, rfield, two_phase_params
from coupled_codefort_2d_b200 import _lib
from coupled_codefort_2d_b200.context import Context, make_params
from coupled_codefort_2d_b200.layout import Grid

pytestmark = pytest.mark.gpu

TOL = 1e-12


def noalloc(L, g, prm, phi, rhs, rho_u, rho_v, tol, max_iter, stream=None, ptrs=None):
    p = make_params(g, prm)
    it, res = C.c_int(-1), C.c_double(-1.0)
    err = C.create_string_buffer(256)
    args = ptrs if ptrs is not None else [_lib.ptr(a) for a in (phi, rhs, rho_u, rho_v)]
    rc = L.fugu_solve_poisson_pressure_noalloc(C.byref(p), stream, *args, float(tol), int(max_iter),
                                               C.byref(it), C.byref(res), err, len(err))
    return rc, it.value, res.value, err.value.decode()


def case(g, seed):
    rng = np.random.default_rng(seed)
    rhs = rfield(rng, g, "cell")
    phi0 = rfield(rng, g, "cell", -0.1, 0.1)
    rho_u = rfield(rng, g, "u", 100.0, 1000.0)
    rho_v = rfield(rng, g, "v", 100.0, 1000.0)
    return phi0, rhs, rho_u, rho_v


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def with_context(g, prm, phi0, rhs, rho_u, rho_v):
    phi = phi0.copy(order="F")
    with Context(g, prm) as ctx:
        it, res = ctx.solve_poisson_pressure(phi, rhs, rho_u, rho_v, 1e-5, 150)
    return phi, it, res


def test_two_calls_in_a_row_match_the_context_entry(gpu):
    L = _lib.lib()
    prm = two_phase_params()
    for name, seed in (("walls_32x24", 21), ("px_16x12", 22)):
        g = GRIDS[name]
        phi0, rhs, rho_u, rho_v = case(g, seed)
        ref_phi, ref_it, ref_res = with_context(g, prm, phi0, rhs, rho_u, rho_v)
        phi = phi0.copy(order="F")
        rc, it, res, msg = noalloc(L, g, prm, phi, rhs, rho_u, rho_v, 1e-5, 150)
        assert rc == 0, msg
        assert it == ref_it
        assert abs(res - ref_res) <= TOL * abs(ref_res)
        assert rel(phi, ref_phi) <= TOL


def test_device_arrays_and_full_size_grid(gpu):
    """Device-memory arguments on a caller's stream, at the largest grid the
    static array holds (256 x 256 cells), twice in a row."""
    import torch

    L = _lib.lib()
    prm = two_phase_params()
    g = Grid(256, 256)
    phi0, rhs, rho_u, rho_v = case(g, 23)
    ref_phi, ref_it, ref_res = with_context(g, prm, phi0, rhs, rho_u, rho_v)
    s = torch.cuda.Stream()
    for _ in range(2):
        # a Fortran-ordered (nx+a, ny+b) array is a C-ordered (ny+b, nx+a) one
        dev = [torch.from_numpy(np.ascontiguousarray(a.T)).cuda() for a in (phi0, rhs, rho_u, rho_v)]
        torch.cuda.synchronize()
        rc, it, res, msg = noalloc(L, g, prm, None, None, None, None, 1e-5, 150,
                                   stream=C.c_void_p(s.cuda_stream), ptrs=[C.c_void_p(t.data_ptr()) for t in dev])
        assert rc == 0, msg
        phi = dev[0].cpu().numpy().T
        assert it == ref_it
        assert abs(res - ref_res) <= TOL * abs(ref_res)
        assert rel(phi, ref_phi) <= TOL


def test_oversize_grid_is_rejected(gpu):
    L = _lib.lib()
    g = Grid(300, 300)
    phi0, rhs, rho_u, rho_v = (g.zeros(k) for k in ("cell", "cell", "u", "v"))
    rc, _, _, msg = noalloc(L, g, two_phase_params(), phi0, rhs, rho_u, rho_v, 1e-5, 150)
    assert rc == -1 and "73728" in msg
