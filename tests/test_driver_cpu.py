"""The fugu2d driver's namelist reader (no GPU needed): the reference's own
input.nml is read with every value of its /sim_params/ group
(input.nml:1-36 of the reference), defaults follow main.f90:55-70 and
mod_params.f90, and malformed input is rejected as Fortran's read(nml=) does."""
import json
import os
import subprocess

import pytest

from conftest import ROOT

# the reference's input.nml, restated as a fixture (values from its /sim_params/ group)
REFERENCE_NML = """&sim_params
  case_type          = 'rising_bubble'
  Lx                 = 1.0d0
  Ly                 = 2.0d0
  Nx_global          = 32
  Ny_global          = 64
  rho1               = 1000.0d0
  rho2               = 100.0d0
  mu1                = 10.0d0
  mu2                = 1.0d0
  sigma              = 24.5d0
  gx                 = 0.0d0
  gy                 = -0.98d0
  dt                 = 2.0d-3
  t_final            = 0.10d0
  cfl_target         = 0.25d0
  max_time_steps     = 100
  time_order         = 2
  tol_bicgstab2      = 1.0d-5
  max_iter_bicgstab2 = 150
  alpha_penalty      = 1.0d12
  periodic_x         = .false.
  periodic_y         = .false.
  adaptive_dt        = .true.
  consistent_amp     = .true.
  use_bicgstab2      = .false.
  restart            = .false.
  vtk_freq           = 20
  chk_freq           = 50
  u_lid              = 1.0d0
  cyl_xc             = 0.5d0
  cyl_yc             = 0.5d0
  cyl_rad            = 0.125d0
  drop_rad           = 0.25d0
  chk_prefix         = 'output/chk_fugu2d'
/
"""


@pytest.fixture(scope="module")
def driver():
    from coupled_codefort_2d_b200 import build

    build.build()
    return build.DRIVER


def run(driver, text, tmp_path):
    p = tmp_path / "input.nml"
    p.write_text(text)
    r = subprocess.run([driver, "--print-params", str(p)], capture_output=True, text=True)
    return r


def test_reads_reference_input_nml(driver, tmp_path):
    r = run(driver, REFERENCE_NML, tmp_path)
    assert r.returncode == 0, r.stderr
    s = json.loads(r.stdout)
    assert s["case_type"] == "rising_bubble" and (s["Nx_global"], s["Ny_global"]) == (32, 64)
    assert (s["Lx"], s["Ly"], s["rho1"], s["rho2"], s["mu1"], s["mu2"]) == (1.0, 2.0, 1000.0, 100.0, 10.0, 1.0)
    assert (s["sigma"], s["gx"], s["gy"], s["dt"], s["t_final"]) == (24.5, 0.0, -0.98, 2.0e-3, 0.10)
    assert (s["cfl_target"], s["max_time_steps"], s["time_order"]) == (0.25, 100, 2)
    assert (s["tol_bicgstab2"], s["max_iter_bicgstab2"], s["alpha_penalty"]) == (1.0e-5, 150, 1.0e12)
    assert (s["periodic_x"], s["periodic_y"], s["adaptive_dt"], s["consistent_amp"]) == (False, False, True, True)
    assert (s["use_bicgstab2"], s["restart"], s["vtk_freq"], s["chk_freq"]) == (False, False, 20, 50)
    assert (s["u_lid"], s["cyl_xc"], s["cyl_yc"], s["cyl_rad"], s["drop_rad"]) == (1.0, 0.5, 0.5, 0.125, 0.25)
    assert s["chk_prefix"] == "output/chk_fugu2d"


def test_defaults_without_file(driver, tmp_path):
    r = subprocess.run([driver, "--print-params", str(tmp_path / "absent.nml")], capture_output=True, text=True)
    assert r.returncode == 0
    s = json.loads(r.stdout)
    # main.f90:55-70 and mod_params.f90 defaults
    assert s["case_type"] == "rising_bubble" and s["vtk_freq"] == 20 and s["chk_freq"] == 50
    assert s["adaptive_dt"] and s["consistent_amp"] and not s["use_bicgstab2"]
    assert (s["Nx_global"], s["rho1"], s["gy"], s["tol_bicgstab2"]) == (64, 1000.0, -9.81, 1e-6)


def test_comments_commas_and_extensions(driver, tmp_path):
    text = """! a comment line
&SIM_PARAMS case_type = "cavity", Nx_global = 128, Ny_global=128 ! trailing comment
  periodic_x = T, dt = 1.0e-2, precision = 'mixed', limiter = 'superbee', krylov_bc_fix = .true.
/
"""
    r = run(driver, text, tmp_path)
    assert r.returncode == 0, r.stderr
    s = json.loads(r.stdout)
    assert s["case_type"] == "cavity" and s["Nx_global"] == 128 and s["Ny_global"] == 128
    assert s["periodic_x"] is True and s["dt"] == 1e-2
    assert s["precision"] == "mixed" and s["limiter"] == "superbee" and s["krylov_bc_fix"] == 1
    assert (s["pcd_smoother"], s["graphs"]) == ("jacobi", 0)


def test_smoother_and_graph_keys(driver, tmp_path):
    text = """&sim_params
  pcd_smoother = 'RBSOR', pcd_sor_omega = 1.5d0, pcd_sweeps = 6, pcd_sweeps_max = 24, graphs = .true.,
  pcd_visc_scale = 1.0d0, vec_rows = 1
/
"""
    r = run(driver, text, tmp_path)
    assert r.returncode == 0, r.stderr
    s = json.loads(r.stdout)
    assert (s["pcd_smoother"], s["pcd_sor_omega"], s["pcd_sweeps"], s["pcd_sweeps_max"], s["graphs"]) == \
        ("rbsor", 1.5, 6, 24, 1)
    assert s["pcd_visc_scale"] == 1.0 and s["vec_rows"] == 1
    r = run(driver, "&sim_params\n  pcd_smoother = 'gauss'\n/\n", tmp_path)
    assert r.returncode == 2 and "pcd_smoother" in r.stderr


def test_unknown_key_rejected(driver, tmp_path):
    r = run(driver, "&sim_params\n  no_such_key = 3\n/\n", tmp_path)
    assert r.returncode == 2 and "unknown namelist key" in r.stderr
