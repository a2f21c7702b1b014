"""Pins the CPU oracle against every analytic acceptance criterion of the
reference's own validation programs (tests/test_*.f90 of
EL-I-Thiam/COUPLED_CODEFORT_2D).  The reference ships no golden vectors and
its Fortran/MPI toolchain is absent here, so these criteria are the pin.
"""
import pytest

import refcases
from oracle.oracle import Oracle


def test_halo_exchange_criterion():
    # tests/test_halo_exchange.f90:113  L_inf < 1e-13
    assert refcases.halo_exchange(Oracle)["err"] < 1e-13


def test_operators_criteria():
    r = refcases.operators(Oracle)
    assert r["div_err"] < 1e-13  # test_operators.f90:159
    assert r["grad_err"] < 5e-2  # :188
    assert r["visc_err"] < 1.0  # :219
    assert r["matvec_finite"]  # :229-237 ("runs")


def test_static_droplet_criteria():
    r = refcases.static_droplet(Oracle)
    assert r["kappa_err_pct"] < 5.0 and r["f_max"] > 10.0  # test_static_droplet.f90:137


def test_laplace_coupled_criteria():
    r = refcases.laplace_coupled(Oracle)
    # test_laplace_coupled.f90:190
    assert r["laplace_err_pct"] < 5.0 and r["mass_err"] < 1e-6 and r["div"] < 1e-4, r


def test_poiseuille_criteria():
    r = refcases.poiseuille(Oracle)
    assert r["rel_l2"] < 1e-2 and r["linf"] < 5e-3, r  # test_poiseuille_twophase.f90:143


def test_week6_darcy_and_restart(tmp_path):
    r = refcases.week6_darcy(Oracle)
    assert r["u_solid"] < 1e-8 and r["div"] < 1e-4, r  # test_week6_advanced.f90:472
    # part B (:481-508): checkpoint after step 10, two more steps, restart -> diff < 1e-14
    g, prm, st, phi = r["grid"], r["prm"], r["state"], r["phi"]
    o = Oracle(g, prm)
    path = str(tmp_path / "chk_r0000.bin")
    assert o.write_checkpoint(path, 10, 0.1, st) == 0
    ref = {k: a.copy(order="F") for k, a in st.items()}
    for step in (11, 12):
        o.step(ref, 0.01, step, use_bicgstab2=False, phi_s=phi)
    back = {k: a.copy(order="F") for k, a in st.items()}
    rc, step, t = o.read_checkpoint(path, back)
    assert rc == 0 and step == 10 and t == 0.1
    for s in (step + 1, step + 2):
        o.step(back, 0.01, s, use_bicgstab2=False, phi_s=phi)
    diff = max(float(abs(ref[k] - back[k]).max()) for k in ("u_vel", "v_vel"))
    assert diff < 1e-14


@pytest.mark.slow
def test_rising_bubble_criteria():
    r = refcases.rising_bubble(Oracle)
    # test_rising_bubble.f90:187
    assert r["y_cm"] > 0.5 and r["v_rise"] > 0 and r["mass_err"] < 1e-6 and r["div"] < 1e-4, r


@pytest.mark.slow
def test_week6_hysing2_amp_criteria():
    r = refcases.week6_hysing2_amp(Oracle)
    assert r["y_cm"] > 0.5 and r["mass_err"] < 1e-5, r  # test_week6_advanced.f90:592


@pytest.mark.slow
def test_lid_driven_cavity_criteria():
    r = refcases.lid_driven_cavity(Oracle)
    # test_lid_driven_cavity.f90:244
    assert abs(r["u_min"]) > 0.15 and abs(r["v_min"]) > 0.15 and r["div"] < 1e-2, r
