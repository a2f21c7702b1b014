"""Step-level parity: ``advance_coupled_step`` on the GPU against the CPU
oracle for every case family the reference tests exercise (cavity with lid,
static droplet with SVOF/CSF, rising bubble with AMP, periodic two-phase
Poiseuille with BDF2, Darcy cylinder with alpha = 1e12), both Krylov solvers,
and the FP64 / mixed defect-correction forms.

Tolerances (the hot path's parity targets): u, v, p relative L2 <= 1e-8 after
N steps on identical inputs; VOF volume equal to 1e-12 relative.  The plain
FP64 form is in fact checked bit for bit (element-wise kernels without FMA
contraction, order-independent reductions on both sides).
"""
import os
import tempfile

import numpy as np
import pytest

from coupled_codefort_2d_b200 import cases
from coupled_codefort_2d_b200.context import Context
from coupled_codefort_2d_b200.layout import Grid
from coupled_codefort_2d_b200.params import Params

pytestmark = pytest.mark.gpu

STATE = ["u_vel", "v_vel", "p_field", "c_field", "u_prev", "v_prev", "rho_c", "rho_u", "rho_v", "kappa",
         "zeta", "eta", "kappa_curv", "f_sigma_u", "f_sigma_v"]


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def case(name):
    """(grid, params, initial colour, step kwargs, dt, nsteps, phi_s)"""
    if name == "cavity":
        g = Grid(24, 24)
        p = Params(rho1=1.0, rho2=1.0, mu1=0.01, mu2=0.01, sigma=0.0, gx=0.0, gy=0.0, time_order=1,
                   tol_bicgstab2=1e-8, max_iter_bicgstab2=100)
        return g, p, g.full("cell", 1.0), dict(u_top_lid=1.0, use_bicgstab2=False), 1e-2, 3, None
    if name == "droplet":
        g = Grid(32, 32)
        p = Params(rho1=1.0, rho2=0.1, mu1=0.1, mu2=0.01, sigma=1.0, gx=0.0, gy=0.0, time_order=2,
                   tol_bicgstab2=1e-6, max_iter_bicgstab2=100)
        c = cases.circle_fraction(g, 0.5, 0.5, 0.25, inside=1.0, ns=8)
        return g, p, c, dict(use_bicgstab2=False), 1e-4, 3, None
    if name == "bubble_amp":
        g = Grid(16, 32, 1.0, 2.0)
        p = Params(rho1=1000.0, rho2=100.0, mu1=10.0, mu2=1.0, sigma=24.5, gx=0.0, gy=-0.98, time_order=2,
                   tol_bicgstab2=1e-6, max_iter_bicgstab2=100)
        c = cases.initial_colour(g, "rising_bubble")
        return g, p, c, dict(use_bicgstab2=False, consistent_amp=True), 1e-3, 3, None
    if name == "bubble_freeslip":
        # the 1 x 2 rising-bubble box with free-slip side walls (extension flag)
        g = Grid(16, 32, 1.0, 2.0)
        p = Params(rho1=1000.0, rho2=100.0, mu1=10.0, mu2=1.0, sigma=24.5, gx=0.0, gy=-0.98, time_order=2,
                   tol_bicgstab2=1e-6, max_iter_bicgstab2=100, free_slip_x=1)
        c = cases.initial_colour(g, "rising_bubble")
        return g, p, c, dict(use_bicgstab2=False), 1e-3, 3, None
    if name == "poiseuille":
        g = Grid(8, 16, periodic_x=True)
        p = Params(rho1=1.0, rho2=1.0, mu1=1.0, mu2=0.25, sigma=0.0, gx=1.0, gy=0.0, time_order=2,
                   tol_bicgstab2=1e-7, max_iter_bicgstab2=200)
        return g, p, cases.initial_colour(g, "poiseuille"), dict(use_bicgstab2=False), 0.05, 3, None
    if name == "cylinder":
        g = Grid(16, 16, periodic_x=True)
        p = Params(rho1=1.0, rho2=1.0, mu1=0.1, mu2=0.1, sigma=0.0, gx=1.0, gy=0.0, time_order=2,
                   alpha_penalty=1e12, tol_bicgstab2=1e-5, max_iter_bicgstab2=150)
        return g, p, g.full("cell", 1.0), dict(use_bicgstab2=False), 0.01, 3, (0.5, 0.5, 0.15)
    if name == "cavity_b2":
        g = Grid(16, 16)
        p = Params(rho1=1.0, rho2=1.0, mu1=0.01, mu2=0.01, sigma=0.0, gx=0.0, gy=0.0, time_order=1,
                   tol_bicgstab2=1e-10, max_iter_bicgstab2=4)
        return g, p, g.full("cell", 1.0), dict(u_top_lid=1.0, use_bicgstab2=True), 1e-2, 2, None
    raise KeyError(name)


def run_pair(oracle_mod, name, prm_override=None, precision=0, nsteps=None):
    g, p, c0, kw, dt, n, cyl = case(name)
    if prm_override:
        p = p.with_(**prm_override)
    n = nsteps or n
    st_o = oracle_mod.new_state(g, c0, p)
    st_g = {k: a.copy(order="F") for k, a in st_o.items()}
    o = oracle_mod.Oracle(g, p)
    phi = o.cylinder_mask(*cyl) if cyl else None
    hist = []
    with Context(g, p, precision=precision) as ctx:
        for step in range(1, n + 1):
            so = o.step(st_o, dt, step, phi_s=phi, **kw)
            sg = ctx.advance_coupled_step(*[st_g[k] for k in STATE], dt, step,
                                          phi_s_u=None if phi is None else phi[0],
                                          phi_s_v=None if phi is None else phi[1], **kw)
            hist.append((so, sg))
    return g, st_o, st_g, hist


@pytest.mark.parametrize("graphs", [0, 1])
@pytest.mark.parametrize("name", ["cavity", "droplet", "bubble_amp", "bubble_freeslip", "poiseuille", "cylinder",
                                  "cavity_b2"])
def test_step_parity_plain_fp64(gpu, oracle_mod, name, graphs):
    """graphs = 1 replays each BiCGStab / BiCGStab(2) iteration from one
    captured CUDA graph, its iteration index kept on the device."""
    g, st_o, st_g, hist = run_pair(oracle_mod, name, dict(graphs=graphs))
    for so, sg in hist:
        assert sg["iter"] == so.iter, (sg["iter"], so.iter)
        assert sg["pcg_calls"] == so.pcg_calls
        assert sg["svof_iters"] == so.svof_iters
    for k in ("u_vel", "v_vel", "p_field"):
        assert rel(st_g[k], st_o[k]) <= 1e-8, (k, rel(st_g[k], st_o[k]))
    vo = cases.fluid1_volume(g, st_o["c_field"])
    vg = cases.fluid1_volume(g, st_g["c_field"])
    assert abs(vg - vo) <= 1e-12 * max(abs(vo), 1e-300)
    for k in STATE:  # bit-exact plain form
        np.testing.assert_array_equal(st_g[k], st_o[k], err_msg=k)


@pytest.mark.parametrize("name", ["droplet", "poiseuille"])
def test_step_parity_grid_wide_pcg(gpu, oracle_mod, name, monkeypatch):
    """The grid-wide persistent PCG (used when a case does not fit one
    thread-block cluster) gives the same bits as the cluster-resident one."""
    monkeypatch.setenv("FUGU_PCG", "grid")
    g, st_o, st_g, hist = run_pair(oracle_mod, name)
    for k in STATE:
        np.testing.assert_array_equal(st_g[k], st_o[k], err_msg=k)


@pytest.mark.parametrize("name,refine,cap0,swmax,smoother", [
    ("droplet", 1, 0, 0, 0), ("droplet", 2, 0, 0, 0), ("bubble_freeslip", 2, 0, 0, 0), ("droplet", 2, 3, 0, 0),
    ("bubble_freeslip", 2, 2, 0, 0), ("bubble_freeslip", 2, 2, 8, 0), ("droplet", 2, 0, 0, 1),
    ("bubble_freeslip", 2, 2, 8, 1), ("poiseuille", 2, 0, 0, 1), ("droplet", 2, 3, 0, 2),
    ("bubble_freeslip", 2, 2, 8, 2)])
def test_refine_fp64_parity(gpu, oracle_mod, name, refine, cap0, swmax, smoother):
    """FP64 defect correction around BiCGStab (refine 1) or flexible GMRES
    (refine 2): same outer and inner iteration counts as the oracle, and the
    same bits.  cap0 > 0 runs the adaptive PCG cap from a start so low that
    it must grow, swmax > 0 then also the PCD sweeps from 1; both carry
    across the steps on both sides.  smoother 1: the PCD's red-black SOR
    velocity smoother (omega 1.5; the periodic channel wraps its colours).
    smoother 2: the same with every Arnoldi step replayed from a CUDA graph."""
    over = dict(refine=refine, refine_inner_tol=1e-2, refine_max_inner=30, refine_max_outer=30, krylov_bc_fix=1,
                tol_bicgstab2=1e-9, pcg_cap_start=cap0, pcd_smoother=min(smoother, 1), pcd_sor_omega=1.5,
                graphs=int(smoother == 2))
    if swmax:  # a low PCG ceiling, so that the sweeps must grow too
        over.update(pcd_sweeps=1, pcd_sweeps_max=swmax, pcg_max_iter=8)
    g, st_o, st_g, hist = run_pair(oracle_mod, name, over)
    for so, sg in hist:
        assert sg["res"] < 1e-9 and so.res < 1e-9
        assert sg["outer"] == so.outer and sg["iter"] == so.iter
        assert sg["pcg_calls"] == so.pcg_calls
    for k in ("u_vel", "v_vel", "p_field"):
        assert rel(st_g[k], st_o[k]) <= 1e-8, (k, rel(st_g[k], st_o[k]))
    for k in STATE:
        np.testing.assert_array_equal(st_g[k], st_o[k], err_msg=k)


@pytest.mark.parametrize("refine,smoother", [(1, 0), (2, 0), (2, 1)])
@pytest.mark.parametrize("name", ["cavity", "droplet", "bubble_amp", "bubble_freeslip", "cylinder"])
def test_mixed_precision_error_vs_fp64_oracle(gpu, oracle_mod, name, refine, smoother):
    """FP32 inner Krylov+PCD inside FP64 defect correction: every step reaches
    the FP64 true residual tolerance (1e-9 relative), and the coupled state
    (u, v, p) stays within 1e-6 relative L2 of the FP64 oracle solving the
    same steps to the same tolerance; per-field errors are reported.
    smoother 1: both sides smooth the PCD's velocity blocks by red-black SOR
    (omega 1.5)."""
    over = dict(refine=refine, refine_inner_tol=1e-2, refine_max_inner=30, refine_max_outer=40, krylov_bc_fix=1,
                tol_bicgstab2=1e-9, pcd_smoother=smoother, pcd_sor_omega=1.5)
    g, st_o, st_g, hist = run_pair(oracle_mod, name, over, precision=1)
    for so, sg in hist:
        assert sg["res"] < 1e-9, sg
        assert sg["status"] == 0
    # In a closed box the pressure is defined up to a constant (the true
    # residual does not see it): compare p with its interior mean removed.
    from coupled_codefort_2d_b200.layout import at

    def p0(p):
        pi = at(p, "cell", slice(1, g.nx), slice(1, g.ny))
        return pi - pi.mean()

    cmp = {"u_vel": (st_g["u_vel"], st_o["u_vel"]), "v_vel": (st_g["v_vel"], st_o["v_vel"]),
           "p_field": (p0(st_g["p_field"]), p0(st_o["p_field"]))}
    per_field = {k: rel(a, b) for k, (a, b) in cmp.items()}
    num = sum(float(np.sum((a - b) ** 2)) for a, b in cmp.values())
    den = sum(float(np.sum(b ** 2)) for a, b in cmp.values())
    coupled = (num / den) ** 0.5
    assert coupled <= 1e-6, (coupled, per_field)
    vo, vg = cases.fluid1_volume(g, st_o["c_field"]), cases.fluid1_volume(g, st_g["c_field"])
    assert abs(vg - vo) <= 1e-6 * abs(vo), (vg, vo)


@pytest.mark.parametrize("name", ["droplet", "bubble_freeslip"])
def test_pcd_viscous_term_fp64_parity(gpu, oracle_mod, name):
    """The PCD with the viscous (Cahouet-Chabard) Schur term inside the FP64
    defect correction around flexible GMRES, with the red-black SOR smoother
    and CUDA graphs: the oracle's iteration counts and bits."""
    over = dict(refine=2, refine_inner_tol=1e-2, refine_max_inner=30, refine_max_outer=30, krylov_bc_fix=1,
                tol_bicgstab2=1e-9, pcg_cap_start=4, pcd_smoother=1, pcd_sor_omega=1.5, pcd_visc_scale=1.0, graphs=1)
    g, st_o, st_g, hist = run_pair(oracle_mod, name, over)
    for so, sg in hist:
        assert sg["res"] < 1e-9 and so.res < 1e-9
        assert sg["outer"] == so.outer and sg["iter"] == so.iter
    for k in STATE:
        np.testing.assert_array_equal(st_g[k], st_o[k], err_msg=k)


def _device_run(name, over, precision, prof):
    """the case's steps on the GPU alone (device-resident state); returns the
    final state, per-step stats and the launch / PCG profile counters"""
    g, p, c0, kw, dt, n, _ = case(name)
    p = p.with_(**over)
    from oracle import oracle as o  # the initial state only

    st = o.new_state(g, c0, p)
    with Context(g, p, precision=precision) as ctx:
        ctx.upload_state(st)
        ctx.profile(1 if prof else 0)
        opts = ctx.step_opts(**kw)
        stats = [ctx.step(dt, s, opts) for s in range(1, n + 1)]
        counters = ctx.profile(-1)
        out = ctx.download_state(STATE)
    return out, stats, counters


@pytest.mark.parametrize("prof", [False, True])
@pytest.mark.parametrize("precision,refine", [(0, 2), (1, 2), (1, 1)])
@pytest.mark.parametrize("name", ["droplet", "bubble_freeslip"])
def test_graph_replay_is_bitwise(gpu, name, precision, refine, prof):
    """graphs = 1 replays each flexible-GMRES Arnoldi step (refine 2) or
    BiCGStab(2) iteration (refine 1) from a CUDA graph: the same kernels with
    the same arguments, so the same bits, iteration counts and kernel-launch
    count as launching them one by one.  Under flexible GMRES the PCG cap and
    the PCD sweeps start low and adapt, so the graphs are re-captured and
    updated in place mid-run; with profiling on, the graphs carry the PCG
    interval events of the launches they time."""
    over = dict(refine=refine, refine_inner_tol=1e-2, refine_max_inner=30, refine_max_outer=30, krylov_bc_fix=1,
                tol_bicgstab2=1e-9)
    if refine == 2:
        over.update(pcg_cap_start=2, pcd_sweeps=1, pcd_sweeps_max=8, pcg_max_iter=8)
    runs = {gr: _device_run(name, dict(over, graphs=gr), precision, prof) for gr in (0, 1)}
    (s0, h0, c0), (s1, h1, c1) = runs[0], runs[1]
    for a, b in zip(h0, h1):  # the low PCG ceiling may stop a mixed solve short: equal either way
        assert a == b
    for k in STATE:
        np.testing.assert_array_equal(s0[k], s1[k], err_msg=k)
    assert c0["kernel_launches"] == c1["kernel_launches"]
    if prof:
        # launched one by one every PCG launch is timed; replayed, a BiCGStab
        # iteration times all of its launches and a flexible-GMRES cycle the
        # PCG of its first Arnoldi step
        assert c0["pcg_iters_timed"] == c0["pcg_iters"] == c1["pcg_iters"]
        assert c1["pcg_ms"] > 0.0 and c1["pcg_launches"] > 0
        if refine == 1:
            assert (c1["pcg_launches"], c1["pcg_iters_timed"]) == (c0["pcg_launches"], c0["pcg_iters_timed"])
        else:
            assert c1["pcg_launches"] < c0["pcg_launches"]
            assert 0 < c1["pcg_iters_timed"] < c1["pcg_iters"]


@pytest.mark.parametrize("precision,refine", [(0, 2), (1, 2), (1, 1)])
def test_graph_replay_with_grid_wide_pcg(gpu, precision, refine, monkeypatch):
    """The grid-wide PCG (the kernel of cases that do not fit one cluster) is
    captured into the iteration graphs as a cooperative kernel node: the same
    bits, iteration counts and launch count as launching one by one.  With
    profiling on, a replayed flexible-GMRES cycle times only the PCG of its
    first Arnoldi step, so fewer timed launches show that the graphs ran."""
    monkeypatch.setenv("FUGU_PCG", "grid")
    over = dict(refine=refine, refine_inner_tol=1e-2, refine_max_inner=30, refine_max_outer=30, krylov_bc_fix=1,
                tol_bicgstab2=1e-9)
    if refine == 2:
        over.update(pcg_cap_start=2, pcd_sweeps=1, pcd_sweeps_max=8, pcg_max_iter=8)
    runs = {gr: _device_run("droplet", dict(over, graphs=gr), precision, True) for gr in (0, 1)}
    (s0, h0, c0), (s1, h1, c1) = runs[0], runs[1]
    assert c0["pcg_cluster_fp64"] == c0["pcg_cluster_fp32"] == 0
    for a, b in zip(h0, h1):
        assert a == b
    for k in STATE:
        np.testing.assert_array_equal(s0[k], s1[k], err_msg=k)
    assert c0["kernel_launches"] == c1["kernel_launches"]
    assert c0["pcg_iters"] == c1["pcg_iters"]
    if refine == 2:
        assert c1["pcg_launches"] < c0["pcg_launches"]


def test_lean_cluster_pcg_matches_grid_wide(gpu, monkeypatch):
    """A 300 x 384 droplet: 16 CTAs of 24 rows, so each thread of the
    cluster-resident FP32 PCG owns a strip of up to 32 cells, and the lean
    variant (z recomputed from r, p read from shared memory) runs.  The mixed
    form solved to 1e-10 with it and with the grid-wide kernel ends within
    1e-7 of each other (two FP32 inner paths, one FP64 tolerance), and the
    profile shows which PCG ran."""
    from oracle import oracle as o

    g = Grid(300, 384, 1.0, 1.28)
    p = Params(rho1=1.0, rho2=0.1, mu1=0.1, mu2=0.01, sigma=1.0, gx=0.0, gy=0.0, time_order=2,
               tol_bicgstab2=1e-10, max_iter_bicgstab2=500, refine=2, refine_inner_tol=1e-2, refine_max_inner=30,
               refine_max_outer=60, krylov_bc_fix=1, pcg_cap_start=40, pcd_sweeps=6, pcd_sweeps_max=24, graphs=1,
               pcd_visc_scale=1.0)
    c0 = cases.circle_fraction(g, 0.5, 0.64, 0.25, inside=1.0, ns=4)
    out = {}
    for mode in ("cluster", "grid"):
        if mode == "grid":
            monkeypatch.setenv("FUGU_PCG", "grid")
        st = o.new_state(g, c0, p)
        with Context(g, p, precision=1) as ctx:
            ctx.upload_state(st)
            opts = ctx.step_opts(use_bicgstab2=True)
            stats = [ctx.step(1e-4, s, opts) for s in (1, 2)]
            prof = ctx.profile(-1)
            out[mode] = (ctx.download_state(["u_vel", "v_vel", "p_field"]), stats, prof)
    (sc, hc, pc), (sg, hg, pg) = out["cluster"], out["grid"]
    assert pc["pcg_cluster_fp32"] == 16 and pg["pcg_cluster_fp32"] == 0
    assert all(h["status"] == 0 and h["res"] < 1e-10 for h in hc + hg)
    for k in ("u_vel", "v_vel"):
        assert rel(sc[k], sg[k]) <= 1e-7, (k, rel(sc[k], sg[k]))


def test_checkpoint_restart_bitwise(gpu, oracle_mod):
    """mod_io.f90:169-225 format: the GPU writes the reference's byte layout,
    the oracle reads it back, and a restart reproduces the run bit for bit
    (tests/test_week6_advanced.f90:125-156)."""
    g, p, c0, kw, dt, n, cyl = case("cylinder")
    o = oracle_mod.Oracle(g, p)
    phi = o.cylinder_mask(*cyl)
    st0 = oracle_mod.new_state(g, c0, p)
    with tempfile.TemporaryDirectory() as d, Context(g, p) as ctx:
        ctx.upload_state(st0)
        ctx.upload("phi_s_u", phi[0])
        ctx.upload("phi_s_v", phi[1])
        opts = ctx.step_opts(use_bicgstab2=False, penalty=True)
        for s in (1, 2):
            ctx.step(dt, s, opts)
        path = os.path.join(d, "chk_r0000.bin")
        ctx.write_checkpoint(path, 2, 2 * dt)
        st_chk = {k: g.zeros(kd) for k, kd in oracle_mod.STATE_KINDS.items()}
        rc, step, t = o.read_checkpoint(path, st_chk)
        assert rc == 0 and step == 2 and t == 2 * dt
        for k in ("u_vel", "v_vel", "u_prev", "v_prev", "p_field", "c_field"):
            np.testing.assert_array_equal(st_chk[k], ctx.download(k))
        for s in (3, 4):
            ctx.step(dt, s, opts)
        ref = ctx.download_state(["u_vel", "v_vel", "p_field"])
        step, t = ctx.read_checkpoint(path)
        assert step == 2
        for s in (3, 4):
            ctx.step(dt, s, opts)
        for k, a in ref.items():
            np.testing.assert_array_equal(ctx.download(k), a)
