"""The PCD's viscous Schur term (extension, ``pcd_visc_scale``) in the CPU
oracle.  The reference approximates the inverse Schur complement by
-(1/dt + u . grad) A_p^-1 with A_p = -div (1/rho) grad
(``src/mod_pcd_precond.f90:49-64``); the extension adds the viscous
(Cahouet-Chabard) part, -mu z_p.  On a high-density-ratio rising bubble the
flexible-GMRES solve then needs far fewer Arnoldi steps; with the scale 0 the
oracle is the reference's (its golden fixtures are unchanged)."""
from coupled_codefort_2d_b200 import cases
from coupled_codefort_2d_b200.params import Params


def _arnoldi_steps(oracle_mod, spec, visc, nsteps=2):
    g = spec["grid"]
    prm = Params(rho1=spec["rho1"], rho2=spec["rho2"], mu1=spec["mu1"], mu2=spec["mu2"], sigma=spec["sigma"],
                 gx=0.0, gy=-0.98, time_order=2, tol_bicgstab2=1e-8, max_iter_bicgstab2=500, refine=2,
                 refine_inner_tol=1e-2, refine_max_inner=30, refine_max_outer=200, krylov_bc_fix=1, free_slip_x=1,
                 pcg_cap_start=40, pcd_sweeps=6, pcd_sweeps_max=24, pcd_smoother=1, pcd_sor_omega=1.5,
                 pcd_visc_scale=visc)
    c0 = cases.circle_fraction(g, spec["xc"], spec["yc"], spec["radius"], inside=0.0, ns=4)
    st = oracle_mod.new_state(g, c0, prm)
    o = oracle_mod.Oracle(g, prm)
    out = []
    for s in range(1, nsteps + 1):
        r = o.step(st, 5e-4, s, use_bicgstab2=False)
        assert r.res < 1e-8
        out.append(r.iter)
    return out


def test_viscous_schur_term_cuts_arnoldi_steps_on_a_hard_bubble(oracle_mod):
    spec = cases.bubble_ensemble(16)[13]  # 64 x 128, density ratio 794
    assert abs(spec["rho1"] / spec["rho2"] - 794) < 1
    ref = _arnoldi_steps(oracle_mod, spec, 0.0)
    cc = _arnoldi_steps(oracle_mod, spec, 1.0)
    assert cc[1] * 1.5 < ref[1], (ref, cc)  # 36 -> 17 Arnoldi steps in the second step


def test_viscous_schur_term_is_the_stated_formula(oracle_mod):
    """r_p with the term equals r_p without it minus (s * 0.5 * kappa) * z_p,
    cell by cell on the interior, bit for bit (the rest of r_p is unchanged)."""
    import numpy as np

    from conftest import colour, rfield, two_phase_params
    from coupled_codefort_2d_b200.layout import Grid

    g = Grid(13, 9, 1.0, 0.7)
    out = {}
    for s in (0.0, 1.0):
        rng = np.random.default_rng(31)
        prm = two_phase_params(pcd_visc_scale=s)
        o = oracle_mod.Oracle(g, prm)
        pr = o.properties(colour(rng, g))
        z = [rfield(rng, g, k) for k in ("u", "v", "cell")]
        ua, va = rfield(rng, g, "u"), rfield(rng, g, "v")
        r = [g.zeros(k) for k in ("u", "v", "cell")]
        o.pcd(*z, *r, ua, va, pr, 2e-3)
        out[s] = (r[2], z[2], pr["kappa"])
    rp0, zp, kap = out[0.0]
    rp1 = out[1.0][0]
    inner = (slice(2, g.nx + 2), slice(2, g.ny + 2))  # cells 1..nx, 1..ny of the (1-nh) layout
    expect = rp0[inner] - ((1.0 * 0.5) * kap[inner]) * zp[inner]
    np.testing.assert_array_equal(rp1[inner], expect)
