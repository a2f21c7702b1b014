"""C-ABI checks that need no GPU: the in-tree library builds for sm_100a,
loads, exports every entry point ``include/fugu_gpu.h`` declares, its
host-only entries behave, and without a device the API fails loudly with an
error code instead of falling back to the CPU."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "fugu_gpu.h")


@pytest.fixture(scope="module")
def libpath():
    from coupled_codefort_2d_b200 import build

    return build.build()


def header_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\s*\*|unsigned long long)\s+(fugu_\w+)\s*\(", src,
                                 flags=re.M)))


def test_header_declares_the_hot_path_entries():
    fns = header_functions()
    for needed in ("fugu_create", "fugu_step", "fugu_advance_coupled_step", "fugu_matvec_coupled",
                   "fugu_apply_pcd_precond", "fugu_krylov_solve", "fugu_solve_poisson_pressure",
                   "fugu_vof_advection_tvd", "fugu_svof_helmholtz_filter", "fugu_compute_csf_force"):
        assert needed in fns


def test_library_exports_every_header_symbol(libpath):
    out = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(fugu_\w+)", out))
    missing = [f for f in header_functions() if f not in exported]
    assert not missing, missing
    L = C.CDLL(libpath)
    for f in header_functions():
        assert hasattr(L, f)


def test_params_default_matches_reference_constants(libpath):
    from coupled_codefort_2d_b200 import _lib

    p = _lib.FuguParams()
    _lib.lib().fugu_params_default(C.byref(p))
    assert (p.pcg_tol, p.pcg_max_iter, p.pcd_sweeps, p.jacobi_omega) == (1e-5, 150, 3, 0.8)
    assert (p.svof_delta_h, p.svof_max_iter, p.svof_tol) == (1.5, 150, 1e-7)
    assert (p.rho1, p.rho2, p.mu1, p.mu2, p.gy, p.alpha_penalty) == (1000.0, 1.0, 1.0, 0.01, -9.81, 1e12)
    assert p.limiter == 0 and p.refine == 0 and p.krylov_bc_fix == 0 and p.precision == 0


def test_ctypes_structs_match_header_layout():
    """Field order of the ctypes mirrors equals the C struct declarations."""
    from coupled_codefort_2d_b200 import _lib

    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    for cname, py in (("fugu_params", _lib.FuguParams), ("fugu_step_opts", _lib.FuguStepOpts),
                      ("fugu_stats", _lib.FuguStats), ("fugu_batch_opts", _lib.FuguBatchOpts),
                      ("fugu_profile_stats", _lib.FuguProfile)):
        body = re.search(r"typedef struct \{([^}]*)\}\s*" + cname + ";", src).group(1)
        names = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            toks = decl.replace(",", " , ").split()
            for t in toks[1:]:
                if t not in (",", "long", "double", "int"):
                    names.append(t)
        assert names == [n for n, _ in py._fields_], (cname, names)


@pytest.mark.skipif(gpu_available(), reason="checks the no-device error path")
def test_create_without_device_fails_loudly(libpath):
    from coupled_codefort_2d_b200 import _lib
    from coupled_codefort_2d_b200.context import Context
    from coupled_codefort_2d_b200.layout import Grid
    from coupled_codefort_2d_b200.params import Params

    with pytest.raises(_lib.FuguError):
        Context(Grid(8, 8), Params())


def test_invalid_params_rejected_before_any_device_work(libpath):
    from coupled_codefort_2d_b200 import _lib

    L = _lib.lib()
    p = _lib.FuguParams()
    L.fugu_params_default(C.byref(p))
    h = C.c_void_p()
    p.nx = 2  # below the minimum grid
    assert L.fugu_create(C.byref(p), 0, C.byref(h)) == -1
    L.fugu_params_default(C.byref(p))
    p.precision = 1  # mixed precision requires refine = 1
    assert L.fugu_create(C.byref(p), 0, C.byref(h)) == -1
    for bad in (-2, 2):  # vec_rows takes -1, 0 or 1
        L.fugu_params_default(C.byref(p))
        p.vec_rows = bad
        assert L.fugu_create(C.byref(p), 0, C.byref(h)) == -1
    assert L.fugu_create(None, 0, C.byref(h)) == -1
    assert not h.value


def test_missing_library_raises(monkeypatch, tmp_path):
    from coupled_codefort_2d_b200 import _lib

    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.lib()


def test_layout_shapes_match_fortran_bounds():
    from coupled_codefort_2d_b200.layout import Grid, at

    g = Grid(7, 5)
    assert g.shape("cell") == (11, 9) and g.shape("u") == (12, 9)
    assert g.shape("v") == (11, 10) and g.shape("vert") == (12, 10)
    a = g.zeros("u")
    a[0, 0] = 1.0  # the lower-bound element u(0-nh, 1-nh) is the first in memory
    assert at(a, "u", -2, -1) == 1.0 and a.ravel(order="F")[0] == 1.0
    np.testing.assert_array_equal(at(a, "u", slice(0, 7), 3).shape, (8,))


FORTRAN = os.path.join(ROOT, "fortran", "mod_fugu_gpu.f90")
PATCH = os.path.join(ROOT, "fortran", "use_gpu.patch")


def header_struct_fields(cname):
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef struct \{([^}]*)\}\s*" + cname + ";", src).group(1)
    c_names = []
    for decl in body.split(";"):
        toks = decl.replace(",", " , ").split()
        c_names += [t for t in toks[1:] if t not in (",", "long", "double", "int")]
    return c_names


def fortran_source():
    """mod_fugu_gpu.f90 without comments, continuation lines joined"""
    lines = [ln.split("!", 1)[0].rstrip() for ln in open(FORTRAN).read().splitlines()]
    return re.sub(r"&\s*\n\s*", " ", "\n".join(lines))


@pytest.mark.parametrize("cname", ["fugu_params", "fugu_step_opts", "fugu_stats"])
def test_fortran_binding_matches_header_layout(cname):
    """The bind(C) types of the Fortran bridge module fortran/mod_fugu_gpu.f90
    declare the C structs' fields in the same order."""
    ftype = re.search(r"type, bind\(C\) :: " + cname + r"\n(.*?)end type", fortran_source(), flags=re.S).group(1)
    f_names = []
    for line in ftype.splitlines():
        if "::" in line:
            f_names += [n.strip() for n in line.split("::", 1)[1].split(",") if n.strip()]
    assert f_names == header_struct_fields(cname)


def test_fortran_interfaces_bind_header_entries():
    """Every bind(C) procedure of the bridge names an entry of the header and
    takes as many arguments as the C declaration."""
    src = fortran_source()
    hdr = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    binds = re.findall(r"(?:function|subroutine)\s+(\w+)\s*\(([^)]*)\)\s*bind\(C,\s*name=\"(\w+)\"\)", src)
    assert {b[2] for b in binds} >= {"fugu_create", "fugu_advance_coupled_step", "fugu_destroy", "fugu_last_error"}
    for fname, args, cname in binds:
        assert fname == cname
        decl = re.search(r"\b" + cname + r"\s*\(([^)]*)\)\s*;", hdr, flags=re.S)
        assert decl, cname
        c_args = [a for a in decl.group(1).split(",") if a.strip() and a.strip() != "void"]
        f_args = [a for a in args.split(",") if a.strip()]
        assert len(f_args) == len(c_args), (cname, f_args, c_args)


def test_use_gpu_patch_only_adds_lines():
    """The patch that wires the bridge into the reference adds lines at stated
    positions and changes none of the reference's own."""
    hunks = 0
    files = set()
    for ln in open(PATCH).read().splitlines():
        if ln.startswith("+++ b/"):
            files.add(ln[6:])
        elif ln.startswith("@@"):
            m = re.match(r"@@ -(\d+),0 \+(\d+)(?:,(\d+))? @@$", ln)
            assert m, ln
            hunks += 1
        elif files and ln and ln[0] == "-" and not ln.startswith("--- a/"):
            raise AssertionError("removes a reference line: " + ln)
    assert files == {"src/main.f90", "src/mod_solver_coupled.f90", "Makefile"}
    assert hunks == 7
