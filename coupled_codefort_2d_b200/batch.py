"""Batched form: many independent cases advanced together on one GPU.

:class:`Batch` wraps ``fugu_batch_*`` of the C ABI.  Every case is a full
context on the device (its own state, work space and stream); the library
autotunes the thread-block-cluster size of each case's PCG at creation.  By
default a pool of host threads steps the cases, largest grid first; with
``lockstep=True`` the coupled solves of a group of cases advance together, one
launch per kernel family serving every case of the group still running, with
the same results per case.  The groups (cases of one PCG grid class, at most
``lockstep_group`` of them; 0: no limit) run side by side, each on its own
stream and host thread.  The reference runs one case per ``mpirun`` and has no
counterpart.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib, cases
from ._lib import FIELD_KIND, FuguBatchOpts, FuguError, FuguParams, FuguStats, FuguStepOpts
from .context import Context, make_params
from .layout import Grid
from .params import Params

STATE_FIELDS = ("u_vel", "v_vel", "p_field", "c_field", "u_prev", "v_prev", "rho_c", "rho_u", "rho_v", "kappa",
                "zeta", "eta", "kappa_curv", "f_sigma_u", "f_sigma_v")


class Batch:
    """``cases``: a list of ``(Grid, Params, precision)``."""

    def __init__(self, specs, device: int = 0, nthreads: int = 0, max_cluster: int = 0, max_coop: int = 0,
                 lockstep: bool = False, lockstep_group: int = 0):
        self.L = _lib.lib()
        self.specs = list(specs)
        n = len(self.specs)
        arr = (FuguParams * n)(*[make_params(g, prm, prec) for g, prm, prec in self.specs])
        opts = FuguBatchOpts(nthreads, max_cluster, max_coop, int(lockstep), int(lockstep_group))
        h = C.c_void_p()
        rc = self.L.fugu_batch_create(arr, n, int(device), C.byref(opts), C.byref(h))
        if rc != 0:
            raise FuguError(rc, "fugu_batch_create failed (see stderr)")
        self.h = h
        self._views = {}

    def __len__(self):
        return len(self.specs)

    def close(self):
        if getattr(self, "h", None):
            for v in self._views.values():
                v.h = None
            self.L.fugu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def case(self, i: int) -> Context:
        """Non-owning :class:`Context` of case ``i`` (upload, download, profile, routines)."""
        if i not in self._views:
            h = C.c_void_p()
            if self.L.fugu_batch_case(self.h, int(i), C.byref(h)) != 0:
                raise IndexError(i)
            g, prm, prec = self.specs[i]
            self._views[i] = Context.view(h, g, prm, prec)
        return self._views[i]

    def stream_handle(self) -> int:
        """cudaStream_t of the batch: events recorded on it around
        :meth:`run` bracket all of the run's device work."""
        h = C.c_void_p()
        rc = self.L.fugu_batch_get_stream(self.h, C.byref(h))
        if rc != 0:
            raise FuguError(rc, "fugu_batch_get_stream")
        return h.value or 0

    def launches(self) -> int:
        """Kernel launches issued by the batch so far (graph replays included)."""
        return int(self.L.fugu_batch_launches(self.h))

    def run(self, nsteps: int, dt, step0, opts) -> dict:
        """Advance every case ``nsteps`` steps (``dt``, ``step0`` scalars or
        per-case sequences; ``opts`` one :class:`FuguStepOpts` or a list).
        Returns per case the last step's statistics, the run's summed
        statistics (``total``), the largest residual and the status."""
        n = len(self)
        dts = (C.c_double * n)(*np.broadcast_to(np.asarray(dt, dtype=np.float64), (n,)))
        s0 = (C.c_int * n)(*np.broadcast_to(np.asarray(step0, dtype=np.int64), (n,)).tolist())
        ol = opts if isinstance(opts, (list, tuple)) else [opts] * n
        oa = (FuguStepOpts * n)(*ol)
        last = (FuguStats * n)()
        mres = (C.c_double * n)()
        status = (C.c_int * n)()
        total = (FuguStats * n)()
        rc = self.L.fugu_batch_run(self.h, int(nsteps), dts, s0, oa, last, mres, status, total)
        out = {"last": [s.as_dict() for s in last], "total": [s.as_dict() for s in total], "max_res": list(mres),
               "status": list(status)}
        if rc != 0:
            raise FuguError(rc, self.L.fugu_batch_last_error(self.h).decode())
        return out


def initial_bubble_state(ctx: Context, spec: dict) -> None:
    """Upload the rising-bubble initial state of one ensemble case: binary
    colour (``main.f90:137-150``), zero velocity and pressure, properties
    from the colour."""
    g = spec["grid"]
    c0 = cases.binary_circle(g, spec["xc"], spec["yc"], spec["radius"], inside=0.0)
    st = {k: g.zeros(FIELD_KIND[k]) for k in STATE_FIELDS}
    st["c_field"][...] = c0
    ctx.compute_mixture_densities(st["c_field"], st["rho_c"], st["rho_u"], st["rho_v"])
    ctx.compute_mixture_viscosities(st["c_field"], st["kappa"], st["zeta"], st["eta"])
    for k in STATE_FIELDS:
        ctx.upload(k, st[k])


def ensemble_params(spec: dict, **solver) -> Params:
    """Physics of an ensemble case plus the caller's solver settings (BDF2)."""
    kw = dict(rho1=spec["rho1"], rho2=spec["rho2"], mu1=spec["mu1"], mu2=spec["mu2"], sigma=spec["sigma"],
              gx=spec["gx"], gy=spec["gy"], time_order=2, free_slip_x=1)
    kw.update(solver)
    return Params(**kw)
