"""Sharding the batched ensemble over ranks, without a GPU: the partition
covers every case exactly once and balances cells, and a world-size-2 gloo
run of the host logic (shard, barrier, max-reduce of the time, gather of
per-case rows to rank 0) reassembles the whole ensemble.  The GPU stepping
is replaced by a runner that returns per-case rows."""
import json
import os
import socket
import time

import pytest
import torch.multiprocessing as mp

from coupled_codefort_2d_b200 import cases
from coupled_codefort_2d_b200.ensemble import case_cost, partition, run_ensemble


def test_partition_covers_every_case_once_and_balances():
    specs = cases.bubble_ensemble(256)
    costs = [case_cost(s) for s in specs]
    for world in (1, 2, 3, 4, 8):
        shards = partition(costs, world)
        assert len(shards) == world
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(256))
        loads = [sum(costs[i] for i in s) for s in shards]
        # greedy LPT: max load <= mean + the largest single case
        assert max(loads) <= sum(costs) / world + max(costs)
    assert partition(costs, 4) == partition(costs, 4)  # deterministic: no exchange needed


def test_partition_more_ranks_than_cases():
    shards = partition([3.0, 1.0], 4)
    assert sorted(i for s in shards for i in s) == [0, 1]
    assert sum(1 for s in shards if not s) == 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_path, ncases):
    import datetime

    import torch.distributed as dist

    from coupled_codefort_2d_b200.ensemble import _dist_ops

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    barrier, max_reduce, gather = _dist_ops()
    specs = cases.bubble_ensemble(ncases)

    def runner(idx):
        yield "ready", None
        t0 = time.perf_counter()
        time.sleep(0.05 * (rank + 1))  # ranks finish at different times
        rows = [{"case": specs[i]["case"], "status": 0, "max_res": 1e-9, "rank": rank} for i in idx]
        yield "done", (rows, time.perf_counter() - t0)

    res = run_ensemble(specs, 5, rank, world, runner, barrier, max_reduce, gather)
    dist.destroy_process_group()
    if rank == 0:
        with open(out_path, "w") as f:
            json.dump(res, f)
    else:
        assert res is None


@pytest.mark.timeout(120)
def test_gloo_two_ranks_reassemble_the_ensemble(tmp_path):
    out = tmp_path / "res.json"
    mp.start_processes(_worker, args=(2, _free_port(), str(out), 12), nprocs=2, join=True, start_method="spawn")
    res = json.loads(out.read_text())
    assert res["world"] == 2 and res["cases"] == 12 and res["steps"] == 5
    assert [r["case"] for r in res["rows"]] == list(range(12))
    assert {r["rank"] for r in res["rows"]} == {0, 1}
    # the timed region is the slower rank's (max over ranks)
    assert res["seconds"] >= 0.1
    assert res["case_steps_per_s"] == pytest.approx(12 * 5 / res["seconds"])


def test_solver_overrides_from_the_command_line():
    import argparse

    from coupled_codefort_2d_b200.ensemble import SOLVER, solver_from_args

    none = argparse.Namespace(smoother=None, omega=None, sweeps=None, sweeps_max=None, graphs=None)
    assert solver_from_args(none) == SOLVER
    assert SOLVER["pcd_smoother"] == 1 and SOLVER["graphs"] == 1
    a = argparse.Namespace(smoother="jacobi", omega=None, sweeps=3, sweeps_max=0, graphs=0)
    s = solver_from_args(a)
    assert (s["pcd_smoother"], s["pcd_sweeps"], s["pcd_sweeps_max"], s["graphs"]) == (0, 3, 0, 0)
    assert s["pcd_sor_omega"] == SOLVER["pcd_sor_omega"] and SOLVER["pcd_sweeps"] == 6  # the default is untouched


def test_solve_bytes_counts_each_kernel_family():
    """The batched roofline's algorithmic bytes, by hand for one step of a
    64 x 128 case: 40 Arnoldi steps in 2 passes (mean j = 9.5), 1000 PCG
    iterations, FP32 inner solve, 6 smoother sweeps."""
    from coupled_codefort_2d_b200.ensemble import solve_bytes
    from coupled_codefort_2d_b200.layout import Grid

    spec = {"grid": Grid(64, 128)}
    n = 64 * 128.0
    n3 = 3 * n
    per_arnoldi = (19 * n + 2 * 6 * 7 * n + 14 * n + (2 * 11.5 + 2 * 12.5 + 4) * n3) * 4
    per_outer = 14 * n * 8 + 4 * n3 * 8 + 12 * n3 + 20 * n3
    want = 40 * per_arnoldi + 9 * n * 4 * 1000 + 2 * per_outer
    got = solve_bytes(spec, [{"iter": 40, "outer": 2, "pcg_iters": 1000}], {"pcd_sweeps": 6}, 4)
    assert abs(got - want) <= 1e-9 * want
