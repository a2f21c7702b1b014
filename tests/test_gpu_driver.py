"""The fugu2d driver end to end on the GPU: an input.nml of the reference's
shape (rising bubble, adaptive dt, AMP, BiCGStab, VTK and checkpoint output)
runs the time loop of main.f90:193-248, and the state it checkpoints is the
oracle's, bit for bit, after the same loop on the CPU (adaptive dt from
compute_adaptive_dt, mod_solver_coupled.f90:41-91, then advance_coupled_step).
The VTK file of the same step holds the oracle's fields, value for value, in
the layout of write_vtk_fields (mod_io.f90:29-164).
"""
import subprocess

import numpy as np
import pytest

from coupled_codefort_2d_b200 import cases
from coupled_codefort_2d_b200.layout import Grid
from coupled_codefort_2d_b200.params import Params

pytestmark = pytest.mark.gpu

NML = """&sim_params
  case_type = 'rising_bubble'
  Lx = 1.0d0, Ly = 2.0d0, Nx_global = 16, Ny_global = 32
  rho1 = 1000.0d0, rho2 = 100.0d0, mu1 = 10.0d0, mu2 = 1.0d0, sigma = 24.5d0
  gx = 0.0d0, gy = -0.98d0
  dt = 2.0d-3, t_final = 1.0d0, cfl_target = 0.25d0, max_time_steps = 4
  time_order = 2, tol_bicgstab2 = 1.0d-6, max_iter_bicgstab2 = 150, alpha_penalty = 1.0d12
  periodic_x = .false., periodic_y = .false., adaptive_dt = .true., consistent_amp = .true.
  use_bicgstab2 = .false., restart = .false.
  vtk_freq = 2, chk_freq = 4, drop_rad = 0.25d0
  chk_prefix = 'output/chk_fugu2d'
/
"""


@pytest.fixture(scope="module")
def driver():
    from coupled_codefort_2d_b200 import build

    build.build()
    return build.DRIVER


def test_driver_run_matches_oracle_loop(gpu, oracle_mod, driver, tmp_path):
    (tmp_path / "input.nml").write_text(NML)
    r = subprocess.run([driver, "input.nml"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Simulation finished" in r.stdout
    for name in ("fugu2d_0000.vtk", "fugu2d_0002.vtk", "fugu2d_0004.vtk", "chk_fugu2d_r0000.bin"):
        assert (tmp_path / "output" / name).exists(), name
    vtk = (tmp_path / "output" / "fugu2d_0004.vtk").read_text()

    g = Grid(16, 32, 1.0, 2.0)
    p = Params(rho1=1000.0, rho2=100.0, mu1=10.0, mu2=1.0, sigma=24.5, gx=0.0, gy=-0.98, cfl_target=0.25,
               time_order=2, tol_bicgstab2=1e-6, max_iter_bicgstab2=150, alpha_penalty=1e12)
    o = oracle_mod.Oracle(g, p)
    st = oracle_mod.new_state(g, cases.initial_colour(g, "rising_bubble", 0.25), p)
    t = 0.0
    for step in range(1, 5):
        dt = o.adaptive_dt(st["u_vel"], st["v_vel"], 2.0e-3)
        dt = min(dt, 1.0 - t)
        o.step(st, dt, step, use_bicgstab2=False, consistent_amp=True)
        t += dt
    chk = {k: g.zeros(kd) for k, kd in oracle_mod.STATE_KINDS.items()}
    rc, step, t_chk = o.read_checkpoint(str(tmp_path / "output" / "chk_fugu2d_r0000.bin"), chk)
    assert rc == 0 and step == 4
    assert t_chk == t
    for k in ("u_vel", "v_vel", "u_prev", "v_prev", "p_field", "c_field"):
        np.testing.assert_array_equal(chk[k], st[k], err_msg=k)
    check_vtk(vtk, g, st)


def fmt(x):
    """the ES15.7 edit descriptor of mod_io.f90:117-152 (C's %15.7E)"""
    return "%15.7E" % x


def check_vtk(text, g, st):
    """The VTK file of mod_io.f90:106-156 written from the oracle's state:
    header, the four cell scalars in i-fastest order, and the cell-centred
    velocity half*(u(i-1,j)+u(i,j)), half*(v(i,j-1)+v(i,j)) (mod_io.f90:47-52),
    every value as the same 15-character field."""
    lines = text.splitlines()
    nx, ny = g.nx, g.ny
    assert lines[:4] == ["# vtk DataFile Version 3.0", "FUGU-2D Coupled Two-Phase Solver Output", "ASCII",
                         "DATASET STRUCTURED_POINTS"]
    assert lines[4] == "DIMENSIONS " + "%8d%8d%8d" % (nx, ny, 1)
    assert lines[5] == "ORIGIN " + fmt(0.5 * g.dx) + fmt(0.5 * g.dy) + fmt(0.0)
    assert lines[6] == "SPACING " + fmt(g.dx) + fmt(g.dy) + fmt(g.dx)
    assert lines[7] == "POINT_DATA %10d" % (nx * ny)
    at = 8
    cell = lambda a, i, j: a[i + 1, j + 1]  # cell (i, j) of a (1-nh:nx+nh, 1-nh:ny+nh) array
    for name, key in (("VOF_C", "c_field"), ("Pressure", "p_field"), ("Density", "rho_c"),
                      ("Curvature", "kappa_curv")):
        assert lines[at:at + 2] == ["SCALARS %s double 1" % name, "LOOKUP_TABLE default"], name
        want = [fmt(cell(st[key], i, j)) for j in range(1, ny + 1) for i in range(1, nx + 1)]
        assert lines[at + 2:at + 2 + nx * ny] == want, name
        at += 2 + nx * ny
    assert lines[at] == "VECTORS Velocity double"
    u, v = st["u_vel"], st["v_vel"]  # u (0-nh:nx+nh, 1-nh:ny+nh), v (1-nh:nx+nh, 0-nh:ny+nh)
    want = [fmt(0.5 * (u[i + 1, j + 1] + u[i + 2, j + 1])) + fmt(0.5 * (v[i + 1, j + 1] + v[i + 1, j + 2])) + fmt(0.0)
            for j in range(1, ny + 1) for i in range(1, nx + 1)]
    assert lines[at + 1:at + 1 + nx * ny] == want
    assert len(lines) == at + 1 + nx * ny


def test_driver_restart_continues_the_run(gpu, driver, tmp_path):
    """restart = .true. reads <chk_prefix>_r0000.bin and continues from its
    step (main.f90:120-131)."""
    (tmp_path / "input.nml").write_text(NML)
    r = subprocess.run([driver, "input.nml"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    (tmp_path / "input.nml").write_text(NML.replace("restart = .false.", "restart = .true.")
                                        .replace("max_time_steps = 4", "max_time_steps = 6"))
    r = subprocess.run([driver, "input.nml"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Restart from step      4" in r.stdout
    assert (tmp_path / "output" / "fugu2d_0006.vtk").exists()
