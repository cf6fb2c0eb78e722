#!/usr/bin/env python
"""Benchmark of the hot path: plain FP32 acoustic leapfrog at 1024^3.

Workload (the acoustic plain-FP32-at-scale configuration): 1024^3 halo-inclusive
grid (1016^3 interior points), seeded layered velocity (8 layers 1500->4500 m/s
with depth, x(1 + 0.05 g), g Gaussian-correlated over 20 cells), dx = 10 m,
dt = 0.4 dx / v_max, 15 Hz Ricker at (512, 512, 16), p = p_prev = 0 at t = 0.
A step is one time step over the whole grid: one launch of the TMA pencil
kernel (in-place leapfrog) with the source injected.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  value = interior point updates per second over
all ranks (Gpts/s); with N > 1 every rank runs an independent replica of the
workload (the path has no exchange step on one grid per GPU), so scaling is weak.
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import re
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_DEFAULT = 1024
DX = 10.0
FREQ = 15.0
SEED = 1234
CONFIG_STEPS = 1000
BYTES_PER_POINT = 16  # read p, p_prev, vel2; write p_next (FP32)
CPU_SAMPLE_NZ = 72    # z-slab of the same grid for the CPU reference timing


def args_():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=N_DEFAULT, help="grid extent per axis (halo incl.)")
    ap.add_argument("--e2e-steps", type=int, default=CONFIG_STEPS)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (heuristic tile)")
    ap.add_argument("--variant", type=int, default=-1, help="force a pencil variant (profiling)")
    ap.add_argument("--zchunks", type=int, default=1)
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def workload(n: int, rank: int = 0):
    import stencil_solver_b200 as sb

    vel2, vmax = sb.model_layered(n, n, n, SEED + rank)
    dt = float(np.float32(0.4 * DX / vmax))
    g = sb.Grid(n, n, n, DX, DX, DX, dt)
    src = g.index(n // 2, n // 2, 16)
    return g, vel2, vmax, src


def workload_desc(n, dt, vmax):
    return {
        "workload": f"acoustic_fp32_{n}^3_layered",
        "grid": [n, n, n],
        "interior_points": (n - 8) ** 3,
        "dx_m": DX, "dt_s": dt, "v_max_mps": round(vmax, 2),
        "source": {"type": "ricker", "freq_hz": FREQ, "cell": [n // 2, n // 2, 16]},
        "model": f"8 layers 1500-4500 m/s x (1+0.05 g), corr 20 cells, seed {SEED}+rank",
        "l2_policy": "inputs larger than L2 (three 4 GiB fields), no flush",
    }


# ── reference CPU path (oracle/_ref) on a bounded sample ───────────────────────

def cpu_reference_sample(n: int, steps: int, warmup: int, seconds: float | None):
    """Times the reference's CPU launch_naive (OpenMP, the reference's Release flags)
    on a z-slab [0, CPU_SAMPLE_NZ) of the same model with the same source, started
    from rest.  Returns (gpts_per_s, cores, sample_text, kind, steps_done)."""
    import oracle
    import stencil_solver_b200 as sb

    variant = "f32" if oracle.ref_available("f32") else None
    nz = CPU_SAMPLE_NZ
    vel2_full, vmax = sb.model_layered(n, n, n, SEED)
    vel2 = np.ascontiguousarray(vel2_full[:nz])
    del vel2_full
    dt = float(np.float32(0.4 * DX / vmax))
    src = (16 * n + n // 2) * n + n // 2
    w = sb.ricker(FREQ, 1.0 / FREQ, dt, 100000)
    p = np.zeros((nz, n, n), np.float32)
    q = np.zeros_like(p)
    interior = (n - 8) * (n - 8) * (nz - 8)

    def one(step_i):
        nonlocal p, q
        if variant:
            oracle.ref_wave_step(p, q, vel2, DX, DX, DX, dt, variant=variant, out=q)
        else:
            oracle.wave_step(p, q, vel2, DX, DX, DX, dt, out=q)
        k = np.float32(np.float32(dt) * np.float32(dt)) * vel2.flat[src]
        q.flat[src] = np.float32(q.flat[src] + np.float32(k * w[step_i]))
        p, q = q, p

    for s in range(warmup):
        one(s)
    t0 = time.perf_counter()
    done = 0
    while True:
        one(warmup + done)
        done += 1
        el = time.perf_counter() - t0
        if seconds is None and done >= steps:
            break
        if seconds is not None and (el >= seconds or done >= max(steps, 1) * 50):
            if done >= 1:
                break
    el = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    kind = "reference" if variant else "port"
    sample = (f"{done} steps of a {n}x{n}x{nz} z-slab (interior {n-8}x{n-8}x{nz-8}) of the "
              f"same layered model and source, from rest; "
              f"{'reference launch_naive CPU path (-O3 -march=x86-64-v4 -fopenmp)' if variant else 'oracle port'}")
    return interior * done / el / 1e9, cores, sample, kind, done, el, dt, vmax


def run_reference(a):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    v, cores, sample, kind, done, el, dt, vmax = cpu_reference_sample(a.n, a.steps, a.warmup,
                                                                       None)
    line = {
        "metric": "acoustic interior grid-point updates per second",
        "value": v, "unit": "Gpts/s", "impl": "reference", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": el / max(done, 1) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": workload_desc(a.n, dt, vmax) | {"sample": sample},
        "cpu_baseline": {"value": v, "unit": "Gpts/s", "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": v, "unit": "Gpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ── clocks and profile summaries ───────────────────────────────────────────────

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        import torch

        self.idx = str(device_index)
        try:  # nvidia-smi numbers GPUs physically; address ours by UUID
            u = str(torch.cuda.get_device_properties(device_index).uuid)
            self.idx = u if u.startswith("GPU-") else "GPU-" + u
        except Exception:  # noqa: BLE001 -- fall back to the index
            pass
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = max(smax, float(r[2]))
                for nm, val in zip(names, r[5:9]):
                    if val.strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback (6.65 TB/s)"


def profiled_traffic_per_point():
    """DRAM bytes per interior point of the pencil kernel from the committed ncu summary."""
    f = ROOT / "profiles" / "wave_pencil_f32_acoustic.md"
    if not f.exists():
        return None
    m = re.search(r"dram_bytes_per_interior_point:\s*([0-9.]+)", f.read_text())
    return float(m.group(1)) if m else None


# ── our arm ───────────────────────────────────────────────────────────────────

def run_ours(a):
    import torch

    import stencil_solver_b200 as sb

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    sb.upload_fd_coefficients()
    n = a.n
    g, vel2, vmax, src = workload(n, rank)
    w = sb.ricker(FREQ, 1.0 / FREQ, g.dt, max(a.e2e_steps, a.steps + a.warmup))
    stream = torch.cuda.current_stream()

    # ── device-resident run: value + roofline ──
    p = torch.zeros(g.shape, dtype=torch.float32, device="cuda")
    q = torch.zeros_like(p)
    v = torch.from_numpy(vel2).cuda()
    step = 0
    tuned = None
    if a.variant >= 0:
        sb.set_pencil_override(sb.KIND_WAVE_F32, a.variant, a.zchunks)
    elif not a.no_tune:  # untimed: pick the tile shape / z split for this grid
        scratch = torch.empty_like(p)
        tuned = sb.tune(sb.KIND_WAVE_F32, g, p, q, v, scratch, reps=5)
        del scratch

    def one():
        nonlocal p, q, step
        sb.wave_step(p, q, v, q, g, src, float(w[step]), stream)
        p, q = q, p
        step += 1

    for _ in range(a.warmup):
        one()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    h0 = time.perf_counter()
    for _ in range(a.steps):
        one()
    host_issue_ms = (time.perf_counter() - h0) * 1e3 / a.steps  # launch cost on the host
    e1.record(stream)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    ms_max = ms
    if pg:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms_max = float(t.item())
    assert sb.device_error() == 0, "device error word set during the timed run"

    ms_step = ms_max / a.steps
    value = world * g.interior * a.steps / (ms_max * 1e-3) / 1e9
    peak, peak_src = measured_peak()
    achieved = BYTES_PER_POINT * g.interior / (ms / a.steps * 1e-3) / 1e9
    tpp = profiled_traffic_per_point()
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_src,
            "traffic": (tpp * g.interior if tpp else None),
            "algorithmic_bytes_per_launch": BYTES_PER_POINT * g.interior,
            "kernel": "pencil_f32_kernel (acoustic)"}
    del p, q
    torch.cuda.empty_cache()

    # ── end to end through the C ABI with host buffers: the whole job ──
    E = a.e2e_steps
    hv = torch.from_numpy(vel2).pin_memory()
    hp = torch.zeros(g.shape, dtype=torch.float32).pin_memory()
    hq = torch.zeros(g.shape, dtype=torch.float32).pin_memory()
    hout = torch.empty(g.shape, dtype=torch.float32).pin_memory()
    htrace = torch.empty(E, dtype=torch.float32).pin_memory()
    dv = torch.empty(g.shape, dtype=torch.float32, device="cuda")
    dp = torch.empty_like(dv)
    dq = torch.empty_like(dv)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    dv.copy_(hv, non_blocking=True)
    dp.copy_(hp, non_blocking=True)
    dq.copy_(hq, non_blocking=True)
    for s in range(E):
        sb.wave_step(dp, dq, dv, dq, g, src, float(w[s]), stream)
        dp, dq = dq, dp
        htrace[s:s + 1].copy_(dp.view(-1)[src:src + 1], non_blocking=True)  # per-step D2H
    hout.copy_(dp, non_blocking=True)
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1)
    if pg:
        t = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_ms = float(t.item())
    assert np.isfinite(htrace.numpy()).all()
    h2d = 3 * g.size * 4 + 0  # vel2, p, p_prev (the per-step source sample is a kernel argument)
    d2h = g.size * 4 + E * 4  # final field + one trace sample per step
    e2e = {"value": world * g.interior * E / (e2e_ms * 1e-3) / 1e9, "unit": "Gpts/s",
           "h2d_bytes_per_step": h2d / E, "d2h_bytes_per_step": d2h / E,
           "steps": E, "ms_total": e2e_ms,
           "api": "sb200_wave_step_f32 per step; fields uploaded from / downloaded to pinned "
                  "host memory inside the timed region; centre trace recorded every step"}
    del dv, dp, dq, hv, hp, hq
    torch.cuda.empty_cache()

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cv, cores, sample, kind, *_ = cpu_reference_sample(n, 1, 2, a.cpu_seconds)
        cpu = {"value": cv, "unit": "Gpts/s", "cores": cores, "kind": kind, "sample": sample}

    choice = sb.pencil_choice(sb.KIND_WAVE_F32, g)
    vname = sb.variant_names()[choice[0]]
    line = {
        "metric": "acoustic interior grid-point updates per second",
        "value": value, "unit": "Gpts/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_desc(n, g.dt, vmax) | {"parallelism": f"replicas{world}",
                                               "tile": vname, "zchunks": choice[1],
                                               "tuned": tuned is not None},
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
        "gpu_launches": a.steps,
        "host_issue_ms_per_step": host_issue_ms,
    }
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    a = args_()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
