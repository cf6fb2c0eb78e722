"""The bench's multi-rank bookkeeping on CPU: two gloo ranks (replicas) agree
on the slowest rank's time, and the whole-job figure counts every rank's
points over that time."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow replica
        out[rank] = bench.max_over_ranks(dist, ms, device="cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        got = dict(out)
    assert got == {0: 15.0, 1: 15.0}


def test_job_throughput_counts_every_rank():
    assert bench.max_over_ranks(None, 12.5) == 12.5
    one = bench.job_gpts(1, 1_000_000_000, 10, 20.0)
    assert one == pytest.approx(500.0)
    assert bench.job_gpts(4, 1_000_000_000, 10, 20.0) == pytest.approx(4 * one)


def test_time_to_solution_summary():
    sec = {"fp16_storage": {"ms_per_step": 1.62,
                            "accuracy_256^3_500_steps": {"field_rel_l2_vs_fp32": 0.018,
                                                         "trace_rel_l2_vs_fp32": 7e-4}},
           "learned": {"coarse_steps": 200, "fine_ms": 1100.0,
                       "judged": {"ms": 110.0, "fallback_at_step": None, "rel_l2": 3e-4,
                                  "speedup_vs_fine": 10.0}}}
    s = bench.time_to_solution_summary(2.72, sec)
    assert s["plain_fp32_1024^3_1000_steps_ms"] == pytest.approx(2720.0)
    assert s["fp16_1024^3_1000_steps_ms"] == pytest.approx(1620.0)
    assert not s["fp16_field_within_1e-3"] and s["fp16_trace_within_1e-3"]
    assert s["learned_within_1e-3"] and s["learned_speedup_vs_fine"] == 10.0
    assert s["learned_coarse_steps"] == 200 and s["learned_judged_ms"] == 110.0
    sec["learned"]["judged"]["fallback_at_step"] = 100  # the judge fell back
    assert not bench.time_to_solution_summary(2.72, sec)["learned_within_1e-3"]
    assert bench.time_to_solution_summary(2.72, {}) == {"plain_fp32_1024^3_1000_steps_ms": 2720.0}


def test_reference_arm_loads_only_the_oracle():
    """bench.py --impl reference times the reference's CPU path through oracle/
    alone: the process never imports the product package nor maps its library,
    and its config is the workload description our arm prints."""
    import json
    import subprocess
    import sys

    code = (
        "import sys, runpy\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--n', '48', '--steps', '2',"
        " '--warmup', '1']\n"
        "runpy.run_path('bench.py', run_name='__main__')\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('LOADED', 'libstencil_b200' in maps, 'stencil_solver_b200' in sys.modules)\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=str(bench.ROOT), capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    assert lines[-1] == "LOADED False False"
    line = json.loads(lines[-2])
    assert line["impl"] == "reference" and line["steps"] == 2 and line["value"] > 0
    assert line["config"] == bench.workload_desc(48, line["config"]["dt_s"],
                                                 line["config"]["v_max_mps"])
    assert line["cpu_baseline"]["cores"] >= 1 and line["e2e"]["h2d_bytes_per_step"] == 0
