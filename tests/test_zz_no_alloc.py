"""The allocation-free Poisson entry, fugu_solve_poisson_pressure_noalloc,
checked against the oracle's solve_poisson_pressure on the same inputs.

Some callers cannot allocate device memory: a host code whose own pool
allocator already holds the device, or a time loop that cannot take the
device-wide synchronisation of cudaFree.  The entry runs the grid-wide PCG
kernel on one static device array instead.  Both the kernel and the oracle
accumulate the PCG scalars error-free, so the tolerance here (the same
iteration count, 1e-12 relative on phi and on the residual) is far above what
the two can differ by.  Two calls in a row (two different cases) check that
nothing of one call leaks into the next, and the device's free memory
(cudaMemGetInfo) must not move across a call once the library is loaded.

This file is collected last on purpose: the entry must work both in a fresh
process and after every other GPU test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import GRIDS, rfield, two_phase_params
from coupled_codefort_2d_b200 import _lib
from coupled_codefort_2d_b200.context import make_params
from coupled_codefort_2d_b200.layout import Grid

pytestmark = pytest.mark.gpu

TOL = 1e-12
FUGU_EINVAL, FUGU_ETIMEOUT = -1, -5


def noalloc(L, g, prm, phi, rhs, rho_u, rho_v, tol, max_iter, stream=None, ptrs=None):
    p = make_params(g, prm)
    it, res = C.c_int(-1), C.c_double(-1.0)
    err = C.create_string_buffer(256)
    args = ptrs if ptrs is not None else [_lib.ptr(a) for a in (phi, rhs, rho_u, rho_v)]
    rc = L.fugu_solve_poisson_pressure_noalloc(C.byref(p), stream, *args, float(tol), int(max_iter),
                                               C.byref(it), C.byref(res), err, len(err))
    return rc, it.value, res.value, err.value.decode()


def case(o, g, seed):
    """rhs, initial phi and the face densities of a seeded two-phase colour
    field (densities 1000 / 100), through the oracle's mixture law."""
    rng = np.random.default_rng(seed)
    c = np.asfortranarray(rng.uniform(0.0, 1.0, size=g.shape("cell")))
    pr = o.properties(c)
    rhs = rfield(rng, g, "cell")
    phi0 = rfield(rng, g, "cell", -0.1, 0.1)
    return phi0, rhs, pr["rho_u"], pr["rho_v"]


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def with_oracle(o, phi0, rhs, rho_u, rho_v):
    phi = phi0.copy(order="F")
    it, res = o.poisson(phi, rhs, rho_u, rho_v, 1e-5, 150)
    return phi, it, res


def check(phi, it, res, ref):
    ref_phi, ref_it, ref_res = ref
    assert it == ref_it
    assert abs(res - ref_res) <= TOL * abs(ref_res)
    assert rel(phi, ref_phi) <= TOL


def test_two_calls_in_a_row_match_the_oracle(gpu, oracle_mod):
    L = _lib.lib()
    prm = two_phase_params()
    for name, seed in (("walls_32x24", 21), ("px_16x12", 22)):
        g = GRIDS[name]
        o = oracle_mod.Oracle(g, prm)
        phi0, rhs, rho_u, rho_v = case(o, g, seed)
        ref = with_oracle(o, phi0, rhs, rho_u, rho_v)
        phi = phi0.copy(order="F")
        rc, it, res, msg = noalloc(L, g, prm, phi, rhs, rho_u, rho_v, 1e-5, 150)
        assert rc == 0, msg
        check(phi, it, res, ref)


def test_device_arrays_full_size_grid_and_no_allocation(gpu, oracle_mod):
    """Device-memory arguments on a caller's stream, at the largest grid the
    static array holds (256 x 256 cells), three calls in a row.  The first
    call may load the library's device code (and with it the static array);
    after it the device's free memory stays exactly the same."""
    import torch

    L = _lib.lib()
    prm = two_phase_params()
    g = Grid(256, 256)
    o = oracle_mod.Oracle(g, prm)
    phi0, rhs, rho_u, rho_v = case(o, g, 23)
    ref = with_oracle(o, phi0, rhs, rho_u, rho_v)
    s = torch.cuda.Stream()
    # a Fortran-ordered (nx+a, ny+b) array is a C-ordered (ny+b, nx+a) one
    host = [np.ascontiguousarray(a.T) for a in (phi0, rhs, rho_u, rho_v)]
    dev = [torch.from_numpy(a).cuda() for a in host]
    ptrs = [C.c_void_p(t.data_ptr()) for t in dev]
    torch.cuda.synchronize()
    free = []
    for call in range(3):
        dev[0].copy_(torch.from_numpy(host[0]))  # phi is intent(inout): the same initial guess each time
        torch.cuda.synchronize()
        rc, it, res, msg = noalloc(L, g, prm, None, None, None, None, 1e-5, 150, stream=C.c_void_p(s.cuda_stream),
                                   ptrs=ptrs)
        assert rc == 0, msg
        free.append(torch.cuda.mem_get_info()[0])
        check(dev[0].cpu().numpy().T, it, res, ref)
    assert free[1] == free[0] and free[2] == free[0], free


def test_oversize_grid_is_rejected(gpu):
    L = _lib.lib()
    g = Grid(300, 300)
    phi0, rhs, rho_u, rho_v = (g.zeros(k) for k in ("cell", "cell", "u", "v"))
    rc, _, _, msg = noalloc(L, g, two_phase_params(), phi0, rhs, rho_u, rho_v, 1e-5, 150)
    assert rc == FUGU_EINVAL and "73728" in msg


def test_barrier_timeout_is_reported_and_the_next_call_recovers(gpu, oracle_mod):
    """The test hook makes the next call's grid barriers wait for one CTA
    more than the launch has; each wait gives up after 1000 polls, so the
    call returns FUGU_ETIMEOUT with a message instead of hanging, and the
    next call solves to the oracle's result."""
    L = _lib.lib()
    prm = two_phase_params()
    g = GRIDS["walls_32x24"]
    o = oracle_mod.Oracle(g, prm)
    phi0, rhs, rho_u, rho_v = case(o, g, 24)
    ref = with_oracle(o, phi0, rhs, rho_u, rho_v)
    assert L.fugu_test_arm_barrier_timeout(None, 1000) == 0
    rc, _, _, msg = noalloc(L, g, prm, phi0.copy(order="F"), rhs, rho_u, rho_v, 1e-5, 150)
    assert rc == FUGU_ETIMEOUT and "gave up" in msg, (rc, msg)
    phi = phi0.copy(order="F")
    rc, it, res, msg = noalloc(L, g, prm, phi, rhs, rho_u, rho_v, 1e-5, 150)
    assert rc == 0, msg
    check(phi, it, res, ref)
