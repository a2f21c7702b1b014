"""bench.py's host-side arithmetic, without a GPU: the roofline figures from
the profile counters, the clock summary from nvidia-smi samples, and the
solver settings of the measured forms."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_roofline_uses_the_timed_launches():
    # 4 timed PCG launches of 40 iterations, 0.2 ms each, on 256^2 cells;
    # all launches together ran 2240 iterations
    prof = {"pcg_launches": 4, "pcg_ms": 0.8, "pcg_iters": 2240, "pcg_iters_timed": 160, "pcg_cells": 65536}
    r = bench.roofline(prof, {"hbm_gbs": 7000.0})
    bytes_per_launch = 9 * 4 * 65536 * 40  # the fused PCG iteration's 9 values per cell
    assert r["bytes_per_launch"] == bytes_per_launch
    assert abs(r["ms_per_launch"] - 0.2) < 1e-12
    assert abs(r["achieved"] - bytes_per_launch / 0.2e-3 / 1e9) < 1e-9
    assert r["peak"] == 7000.0 and r["peak_source"] == "measured"
    assert abs(r["frac"] - r["achieved"] / 7000.0) < 1e-12
    assert r["iters_per_launch"] == 40 and r["timed_launches"] == 4
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"
    # no measured peaks: the fallback copy figure
    assert bench.roofline(prof, None)["peak_source"] == "fallback"
    assert bench.roofline({"pcg_launches": 0}, None) is None


def test_clock_summary_flags_throttle_reasons():
    s = bench.ClockSampler(0)
    s.out = "\n".join([
        "0, 1965, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 980.0, 0x4, Not Active, Not Active, Not Active, Active",
        "0, 300, 1965, 90.0, 0x0, Not Active, Not Active, Not Active, Not Active",
    ])
    r = s.summary()
    assert r["sm_max_mhz"] == 1965.0 and r["samples"] == 3
    assert r["sm_mhz"] == 1957.5  # median of the loaded samples (> half of max)
    assert r["reasons"] == ["sw_power_cap"]


def test_measured_forms_solver_settings():
    mixed = bench.case_params(2)
    assert (mixed.refine, mixed.graphs, mixed.pcg_cap_start, mixed.pcd_sweeps, mixed.pcd_sweeps_max) == \
        (2, 1, 80, 6, 24)
    assert mixed.tol_bicgstab2 == bench.TOL == 1e-8
    assert mixed.pcd_smoother == 0  # the bench keeps the reference's damped Jacobi
    assert mixed.pcd_visc_scale == 1.0  # the headline carries the viscous Schur term
    r = bench.reference_pcd_params(mixed)  # the arm with the reference's PCD
    assert (r.pcd_visc_scale, r.pcg_cap_start, r.refine, r.graphs, r.tol_bicgstab2) == (0.0, 40, 2, 1, 1e-8)
    b2 = bench.case_params(1)  # BiCGStab(2) inner solve: the reference's fixed PCD
    assert (b2.pcd_visc_scale, b2.pcg_cap_start, b2.pcd_sweeps) == (0.0, 0, 3)


def test_reference_toolchain_probe():
    """The reference arm records, on the host it runs on, whether the Fortran
    and MPI tools the reference needs exist (this container has none)."""
    import shutil

    tc = bench.reference_toolchain()
    assert set(tc) == {"gfortran", "mpifort", "mpirun", "cores"} and tc["cores"] >= 1
    for t in ("gfortran", "mpifort", "mpirun"):
        assert tc[t] == shutil.which(t)
