"""Run the benchmark configurations and print their reports (one JSON object
per configuration).

    python -m coupled_codefort_2d_b200.configs c1            # lid-driven cavity, 128^2, 200 steps
    python -m coupled_codefort_2d_b200.configs c2            # static droplet, 256^2, 500 steps
    python -m coupled_codefort_2d_b200.configs c3 --steps N  # rising bubble, 320x640 (6000 steps to t = 3)
    python -m coupled_codefort_2d_b200.configs c4            # 256-case ensemble, 200 steps (the ensemble runner)
    python -m coupled_codefort_2d_b200.configs c5            # adjoint gradients, 160x320, 400 steps
    python -m coupled_codefort_2d_b200.configs scale --n 2048 --steps 1   # droplet at n x n (HBM-bound)

c1: cavity on the unit square, rho = 1, mu = 1e-3 (Re = 1000), lid u = 1, BDF1,
dt = 1e-2, tolerance 1e-10, zero initial fields.  The reference's own solver
cannot reach 1e-10 (its BiCGStab(2) diverges on this case), so the plain FP64
form here is the FP64 defect correction around flexible GMRES + PCD.  Reports
the centreline extremes and the divergence.

c1-c3 run the PCD with the viscous Schur term (PCG cap from 80), c3 also with
the red-black SOR velocity smoother; ``--pcd reference`` runs the reference's
PCD instead.

c2: static droplet (R = 0.25, rho 1 / 0.1, mu 0.1 / 0.01, sigma = 1, no
gravity), area fractions by 16 x 16 sub-sampling, BDF2, dt = 1e-4, 500 steps,
mixed precision and FP64.  Reports the spurious-current max |u|, the pressure
jump against sigma / R (``tests/test_laplace_coupled.f90:129-159``) and mass.

c3: rising bubble in a 1 x 2 box (R = 0.25 at (0.5, 0.5); outer rho 1000,
mu 10; bubble rho 100, mu 1; sigma 24.5; g = 0.98), no-slip top and bottom,
free-slip sides, BDF2, dt = 5e-4; the high-contrast variant has bubble rho 1,
mu 0.1, sigma 1.96.  Mixed precision against FP64: centroid height, rise
velocity (``tests/test_rising_bubble.f90:134-155``) and circularity, and their
differences.

c4: the batched rising-bubble ensemble (256 seeded cases on the grids 64 x 128
to 256 x 512, 200 BDF2 steps each, mixed precision); runs
``python -m coupled_codefort_2d_b200.ensemble --cases 256 --steps N`` and
prints its report (aggregate case-steps/s, per-case failures, max residual).

c5: the discrete adjoint.  Rising bubble (outer rho 1000, mu 10; bubble rho
100, mu 1; sigma 24.5; g = 0.98; area-fraction disc) on 160 x 320, 400 BDF2
steps of dt = 2.5e-3 in FP64 (T = 1), checkpoints every 20 steps; J = the
centroid height at T.  dJ/dsigma, dJ/dmu1 (outer viscosity) and dJ/dC0 for
two interface cells against central differences of the GPU forward run
(h = 1e-6 relative, and 1e-4 for the parameters).  Second check: the steady
two-phase Poiseuille channel, 64 x 128, mu ratio 10, body force 1, against
the analytic derivative of the two-layer profile.

scale: the c2 droplet (BDF2, dt = 1e-4, the bench's solver) on an n x n grid
with n large enough that every field is far larger than the 126 MB L2 (2048^2:
34 MB per FP64 field), so that each kernel of the step streams HBM.  It is the
workload of the per-kernel HBM roofline (ncu launch list of its first step);
colour by 4 x 4 sub-sampling.  Reports steps/s and the device memory held.

Every run is synthetic: the fields are fully determined by the parameters.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import cases
from ._lib import FIELD_KIND, FP64, MIXED
from .context import Context
from .layout import Grid, at
from .params import Params

SOLVER = dict(refine=2, refine_inner_tol=1e-2, refine_max_inner=30, refine_max_outer=60, krylov_bc_fix=1,
              pcg_cap_start=40, pcd_sweeps=6, pcd_sweeps_max=24, graphs=1)
# SOLVER keeps the reference's PCD.  The runs below add (unless --pcd
# reference) the PCD extensions that cut the Arnoldi steps: the viscous Schur
# term with the PCG cap from 80, and on the bubble the red-black SOR smoother.
FAST = dict(pcd_visc_scale=1.0, pcg_cap_start=80)
BUBBLE = dict(FAST, pcd_smoother=1, pcd_sor_omega=1.5)


def solver(args, extra):
    """the solver settings of a run: SOLVER plus the extensions unless --pcd reference"""
    return dict(SOLVER, **({} if getattr(args, "pcd", "fast") == "reference" else extra))
STATE = ("u_vel", "v_vel", "p_field", "c_field", "u_prev", "v_prev", "rho_c", "rho_u", "rho_v", "kappa", "zeta",
         "eta", "kappa_curv", "f_sigma_u", "f_sigma_v")


def _run(g, prm, c0, precision, nsteps, dt, lid=None, every=None, device=0, on_step=None):
    """Advance nsteps from rest; returns the final state, per-step stats and
    seconds of stepping (CUDA-synchronised wall clock)."""
    import torch

    st = {k: g.zeros(FIELD_KIND[k]) for k in STATE}
    st["c_field"][...] = c0
    with Context(g, prm, device=device, precision=precision) as ctx:
        ctx.compute_mixture_densities(st["c_field"], st["rho_c"], st["rho_u"], st["rho_v"])
        ctx.compute_mixture_viscosities(st["c_field"], st["kappa"], st["zeta"], st["eta"])
        ctx.upload_state(st)
        opts = ctx.step_opts(use_bicgstab2=True, u_top_lid=lid)
        stats, hist = [], []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s in range(1, nsteps + 1):
            stats.append(ctx.step(dt, s, opts))
            if every and s % every == 0:
                hist.append((s, ctx.download_state(["c_field", "v_vel"])))
            if on_step:
                on_step(s, ctx)
        torch.cuda.synchronize()
        secs = time.perf_counter() - t0
        out = ctx.download_state(list(STATE))
    return out, stats, secs, hist


def _summary(stats, secs):
    return {"steps_per_s": len(stats) / secs, "max_true_residual": max(s["res"] for s in stats),
            "failed_steps": sum(1 for s in stats if s["status"] != 0),
            "mean_inner_iterations": float(np.mean([s["iter"] for s in stats]))}


def config_c1(args):
    n = 128
    g = Grid(n, n)
    prm = Params(rho1=1.0, rho2=1.0, mu1=1e-3, mu2=1e-3, sigma=0.0, gx=0.0, gy=0.0, time_order=1,
                 tol_bicgstab2=1e-10, max_iter_bicgstab2=500, **solver(args, FAST))
    steps = args.steps or 200
    st, stats, secs, _ = _run(g, prm, g.full("cell", 1.0), FP64, steps, 1e-2, lid=1.0, device=args.device)
    u = st["u_vel"]
    v = st["v_vel"]
    # vertical centreline u(x = 0.5, y) and horizontal centreline v(x, y = 0.5)
    uc = at(u, "u", n // 2, slice(1, n))  # u faces at x = 0.5
    vc = at(v, "v", slice(1, n), n // 2)  # v faces at y = 0.5
    return {"config": "c1", "workload": f"lid_driven_cavity_{n}x{n}_Re1000", "steps": steps, "dtype": "f64",
            "solver": solver(args, FAST),
            **_summary(stats, secs), "u_min_vertical_centreline": float(uc.min()),
            "v_min_horizontal_centreline": float(vc.min()), "v_max_horizontal_centreline": float(vc.max()),
            "max_divergence": cases.max_divergence(g, u, v)}


def config_c2(args):
    n = 256
    g = Grid(n, n)
    prm = Params(rho1=1.0, rho2=0.1, mu1=0.1, mu2=0.01, sigma=1.0, gx=0.0, gy=0.0, time_order=2,
                 tol_bicgstab2=1e-8, max_iter_bicgstab2=500, **solver(args, FAST))
    steps = args.steps or 500
    c0 = cases.circle_fraction(g, 0.5, 0.5, 0.25, inside=1.0, ns=16)
    vol0 = cases.fluid1_volume(g, c0)
    rep = {"config": "c2", "workload": f"static_droplet_{n}x{n}", "steps": steps, "sigma_over_R": 1.0 / 0.25,
           "solver": solver(args, FAST)}
    finals = {}
    for name, prec in (("mixed", MIXED), ("fp64", FP64)):
        st, stats, secs, _ = _run(g, prm, c0, prec, steps, 1e-4, device=args.device)
        umax = float(max(np.abs(at(st["u_vel"], "u", slice(1, n - 1), slice(1, n))).max(),
                         np.abs(at(st["v_vel"], "v", slice(1, n), slice(1, n - 1))).max()))
        dp = cases.laplace_jump(g, st["p_field"], 0.25)
        rep[name] = {**_summary(stats, secs), "spurious_max_u": umax, "pressure_jump": dp,
                     "pressure_jump_rel_error": abs(dp - 4.0) / 4.0,
                     "mass_rel_change": abs(cases.fluid1_volume(g, st["c_field"]) - vol0) / vol0}
        finals[name] = st
    rep["mixed_vs_fp64"] = {k: float(np.linalg.norm(finals["mixed"][k] - finals["fp64"][k]) /
                                     max(np.linalg.norm(finals["fp64"][k]), 1e-300)) for k in ("u_vel", "v_vel")}
    return rep


def config_c3(args):
    g = Grid(320, 640, 1.0, 2.0)
    if args.variant == "high_contrast":
        phys = dict(rho1=1000.0, rho2=1.0, mu1=10.0, mu2=0.1, sigma=1.96)
    else:
        phys = dict(rho1=1000.0, rho2=100.0, mu1=10.0, mu2=1.0, sigma=24.5)
    prm = Params(gx=0.0, gy=-0.98, time_order=2, tol_bicgstab2=1e-8, max_iter_bicgstab2=500, free_slip_x=1,
                 **phys, **solver(args, BUBBLE))
    steps = args.steps or 6000
    dt = 5e-4
    c0 = cases.binary_circle(g, 0.5, 0.5, 0.25, inside=0.0)
    every = max(1, steps // 4)
    rep = {"config": "c3", "workload": f"rising_bubble_320x640_{args.variant}", "steps": steps, "t": steps * dt,
           "solver": solver(args, BUBBLE)}
    hists = {}
    for name, prec in (("mixed", MIXED), ("fp64", FP64)):
        st, stats, secs, hist = _run(g, prm, c0, prec, steps, dt, every=every, device=args.device)
        ycm, vr = cases.bubble_centroid_velocity(g, st["c_field"], st["v_vel"])
        rep[name] = {**_summary(stats, secs), "y_centroid": ycm, "rise_velocity": vr,
                     "circularity": cases.circularity(g, st["c_field"]),
                     "bubble_volume": cases.bubble_volume(g, st["c_field"])}
        hists[name] = [(s, cases.bubble_centroid_velocity(g, h["c_field"], h["v_vel"])) for s, h in hist]
    m, f = rep["mixed"], rep["fp64"]
    rep["mixed_vs_fp64"] = {"y_centroid_abs": abs(m["y_centroid"] - f["y_centroid"]),
                            "rise_velocity_rel": abs(m["rise_velocity"] - f["rise_velocity"]) /
                            max(abs(f["rise_velocity"]), 1e-300),
                            "circularity_abs": abs(m["circularity"] - f["circularity"]),
                            "history": [{"step": s, "y_mixed": a[0], "y_fp64": b[0], "v_mixed": a[1], "v_fp64": b[1]}
                                        for (s, a), (_, b) in zip(hists["mixed"], hists["fp64"])]}
    return rep


def _fd_check(ad, fd):
    return {"adjoint": float(ad), "central_difference": float(fd),
            "rel_difference": float(abs(ad - fd) / max(abs(fd), 1e-300))}


def smooth_interface_direction(pb):
    """A smooth perturbation of the initial colour on the interface cells
    (0.02 < C0 < 0.98), zero on pure cells and ghosts, unit maximum: C0 +- h
    times it stays inside (0, 1) for h < 0.02, so no cell crosses the clip."""
    g = pb.g
    ci = at(pb.c0, "cell", slice(1, g.nx), slice(1, g.ny))
    X, Y = cases.cell_centres_interior(g)
    w = ci * (1.0 - ci) * (1.0 + 0.5 * np.cos(2.0 * np.pi * X) * np.sin(np.pi * Y))
    w[(ci <= 0.02) | (ci >= 0.98)] = 0.0
    out = g.zeros("cell")
    at(out, "cell", slice(1, g.nx), slice(1, g.ny))[...] = w / np.max(w)
    return out


def _h_sweep(pb, grads, dc0, hs):
    """Central differences of J at each h against the adjoint: sigma and mu1
    (h relative to the value) and the smooth interface direction of C0 (h
    absolute, the direction's maximum being 1)."""
    out = {}
    for name in ("sigma", "mu1"):
        v0 = pb.phys[name]
        rows = []
        for hr in hs:
            h = hr * v0
            fd = (pb.value(**{name: v0 + h}) - pb.value(**{name: v0 - h})) / (2 * h)
            rows.append({"h_relative": hr, "central_difference": fd,
                         "relative_difference": abs(grads[name] - fd) / abs(fd)})
        out[f"d{name}"] = {"adjoint": float(grads[name]), "sweep": rows}
    d = smooth_interface_direction(pb)
    ad = float(np.sum(dc0 * d))
    rows = []
    for h in hs:
        fd = (pb.value(c0=pb.c0 + h * d) - pb.value(c0=pb.c0 - h * d)) / (2 * h)
        rows.append({"h": h, "central_difference": fd, "relative_difference": abs(ad - fd) / abs(fd)})
    out["dC0_along_smooth_interface_direction"] = {"adjoint": ad, "sweep": rows}
    return out


def config_c5(args):
    from .adjoint import RisingBubble, SteadyPoiseuille, analytic_grad

    if args.sweep:
        # the h sweep at a smaller size (each central difference is two forward runs)
        steps = args.steps or 100
        pb = RisingBubble(80, 160, nsteps=steps, T=steps * 2.5e-3, checkpoint=20, tol=1e-12, device=args.device)
        J, grads, dc0 = pb.value_and_grad()
        return {"config": "c5", "workload": f"rising_bubble_adjoint_80x160_{steps}_steps_h_sweep", "J": J,
                "checks": _h_sweep(pb, grads, dc0, (1e-8, 1e-7, 1e-6, 1e-5, 1e-4, 1e-3))}
    steps = args.steps or 400
    pb = RisingBubble(160, 320, nsteps=steps, T=steps * 2.5e-3, checkpoint=20, tol=1e-12, device=args.device)
    g = pb.g
    rep = {"config": "c5", "workload": f"rising_bubble_adjoint_160x320_{steps}_steps", "steps": steps,
           "dt": pb.dt, "checkpoint_every": pb.checkpoint, "tolerance": pb.tol}
    t0 = time.perf_counter()
    J, grads, dc0 = pb.value_and_grad()
    rep["gradient_seconds"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    J_fwd = pb.value()
    rep["forward_seconds"] = time.perf_counter() - t0
    rep["J_y_centroid"] = J
    rep["J_equals_forward_run"] = J == J_fwd
    rep["gradient"] = {k: float(v) for k, v in grads.items()}
    checks = {}
    for name in ("sigma", "mu1"):
        v0 = pb.phys[name]
        for hr in (1e-6, 1e-4):
            h = hr * v0
            fd = (pb.value(**{name: v0 + h}) - pb.value(**{name: v0 - h})) / (2 * h)
            checks[f"d{name}_h{hr:g}"] = _fd_check(grads[name], fd)
    ci = at(pb.c0, "cell", slice(1, g.nx), slice(1, g.ny))
    di = at(dc0, "cell", slice(1, g.nx), slice(1, g.ny))
    iface = (ci > 0.1) & (ci < 0.9)
    big = np.unravel_index(np.argmax(np.where(iface, np.abs(di), 0.0)), ci.shape)
    other = [tuple(t) for t in np.argwhere(iface)][len(np.argwhere(iface)) // 3]
    for i0, j0 in (big, other):
        k = (int(i0) + 2, int(j0) + 2)  # the cell array's lower bound is -1
        h = 1e-6 * float(pb.c0[k])
        cp, cm = pb.c0.copy(order="F"), pb.c0.copy(order="F")
        cp[k] += h
        cm[k] -= h
        fd = (pb.value(c0=cp) - pb.value(c0=cm)) / (2 * h)
        checks[f"dC0_cell_{int(i0) + 1}_{int(j0) + 1}_h1e-06"] = _fd_check(dc0[k], fd)
    rep["bubble_checks"] = checks
    # the second check: steady two-phase Poiseuille, 64 x 128, mu ratio 10,
    # against the analytic derivative of the two-layer profile
    pp = SteadyPoiseuille(nx=64, ny=128, device=args.device)
    try:
        mu1, mu2 = 1.0, 0.1
        Jp, gp, _ = pp.value_and_grad(mu1, mu2)
        a1, a2 = analytic_grad(mu1, mu2)
        h = 1e-6
        fd1 = (pp.value(mu1 + h * mu1, mu2) - pp.value(mu1 - h * mu1, mu2)) / (2 * h * mu1)
        rep["poiseuille_64x128"] = {
            "mean_velocity": Jp, "dmu1": _fd_check(gp[0], fd1),
            # d/d(mu1/mu2) at fixed mu2 = mu2 d/dmu1
            "d_ratio_adjoint": mu2 * gp[0], "d_ratio_analytic": mu2 * a1,
            "d_ratio_rel_difference": abs(gp[0] - a1) / abs(a1),
            "dmu2_adjoint": gp[1], "dmu2_analytic": a2}
    finally:
        pp.close()
    return rep


def config_scale(args):
    import torch

    n = args.n
    g = Grid(n, n)
    prm = Params(rho1=1.0, rho2=0.1, mu1=0.1, mu2=0.01, sigma=1.0, gx=0.0, gy=0.0, time_order=2,
                 tol_bicgstab2=1e-8, max_iter_bicgstab2=500, vec_rows=args.vec_rows, **SOLVER)
    steps = args.steps or 1
    c0 = cases.circle_fraction(g, 0.5, 0.5, 0.25, inside=1.0, ns=4)
    prec = {"mixed": MIXED, "fp64": FP64}[args.precision]
    free0, total = torch.cuda.mem_get_info(args.device)
    peak = [0]

    def probe(_s, _ctx):
        peak[0] = max(peak[0], free0 - torch.cuda.mem_get_info(args.device)[0])

    _, stats, secs, _ = _run(g, prm, c0, prec, steps, 1e-4, device=args.device, on_step=probe)
    return {"config": "scale", "workload": f"static_droplet_{n}x{n}", "steps": steps, "precision": args.precision,
            "vec_rows": args.vec_rows,
            **_summary(stats, secs), **{k: [s[k] for s in stats] for k in ("outer", "iter", "pcg_calls", "pcg_iters",
                                                                                "svof_iters")},
            "device_bytes_held": peak[0], "device_bytes_total": total}


def main(argv=None):
    ap = argparse.ArgumentParser(description="run a benchmark configuration and print its report")
    ap.add_argument("config", choices=["c1", "c2", "c3", "c4", "c5", "scale"])
    ap.add_argument("--steps", type=int, default=0, help="override the configuration's step count")
    ap.add_argument("--variant", default="standard", choices=["standard", "high_contrast"], help="c3 only")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--pcd", default="fast", choices=["fast", "reference"],
                    help="c1-c3: the PCD extensions (default) or the reference's PCD")
    ap.add_argument("--n", type=int, default=2048, help="scale only: cells per side")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"], help="scale only")
    ap.add_argument("--vec-rows", type=int, default=0, choices=[-1, 0, 1],
                    help="scale only: fugu_params.vec_rows (0: vector row kernels from 2^20 box points)")
    ap.add_argument("--sweep", action="store_true",
                    help="c5 only: central differences over h = 1e-8 .. 1e-3 at 80 x 160 (the plateau)")
    args = ap.parse_args(argv)
    if args.config == "c4":  # the ensemble runner prints its own report
        from . import ensemble

        ensemble.main(["--cases", "256", "--steps", str(args.steps or 200)])
        return
    rep = {"c1": config_c1, "c2": config_c2, "c3": config_c3, "c5": config_c5, "scale": config_scale}[args.config](args)
    print(json.dumps(rep), flush=True)


if __name__ == "__main__":
    main()
