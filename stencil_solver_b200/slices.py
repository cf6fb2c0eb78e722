"""Slice frames of a simulation in the reference's visualisation format.

The format of the reference's slice writer (src/main_slice.cpp:15-19, 106-152;
scripts/reference_slice.py:84-106 writes the same, scripts/make_slice_gif.py:30-36
reads it):

  PREFIX.f32   float32 frames, frame-major; each frame is one XY plane, ny rows
               of nx values (x fastest).  Frame 0 is the initial state, then one
               frame after every `every` steps.
  PREFIX.json  {"nx", "ny", "nz", "plane": "xy", "plane_index", "frames",
               "every", "steps", "dt", "dx", "velocity", "physics", "kernel",
               "dtype": "float32"}

The reference downloads the whole grid for every frame and keeps one plane;
here each frame is Run.plane (sb200_run_get_plane): only the nx * ny floats of
the plane cross to the host.  FP16-storage runs write frames in physical units
(float32), like FP32 runs.
"""
from __future__ import annotations

import json
import pathlib

import numpy as np

META_KEYS = ("nx", "ny", "nz", "plane", "plane_index", "frames", "every", "steps", "dt", "dx",
             "velocity", "physics", "kernel", "dtype")


def write_slices(run, prefix, steps: int, every: int = 5, plane_index: int | None = None,
                 velocity: float = 0.0, physics: str = "wave", kernel: str = "b200-pencil") -> int:
    """Steps `run` (a Run, or anything with .grid, .steps(n) and .plane(z)) for
    `steps` steps from its current state and writes PREFIX.f32 / PREFIX.json;
    returns the number of frames.  As the reference: --every below 1 is an
    error, the plane defaults to nz / 2, and the last frame is the last multiple
    of `every` (steps after it are still taken)."""
    if every < 1:
        raise ValueError("every must be >= 1")
    if steps < 0:
        raise ValueError("steps must be >= 0")
    g = run.grid
    z = g.nz // 2 if plane_index is None else int(plane_index)
    if not 0 <= z < g.nz:
        raise ValueError(f"plane_index {z} outside [0, {g.nz})")
    prefix = str(prefix)
    frames = 0
    buf = np.empty((g.ny, g.nx), np.float32)
    with open(prefix + ".f32", "wb") as out:
        run.plane(z, buf)
        buf.tofile(out)
        frames += 1
        done = 0
        while done < steps:
            k = min(every, steps - done)
            run.steps(k)
            done += k
            if k == every:
                run.plane(z, buf)
                buf.tofile(out)
                frames += 1
    meta = {"nx": int(g.nx), "ny": int(g.ny), "nz": int(g.nz), "plane": "xy", "plane_index": z,
            "frames": frames, "every": int(every), "steps": int(steps), "dt": float(g.dt),
            "dx": float(g.dx), "velocity": float(velocity), "physics": physics, "kernel": kernel,
            "dtype": "float32"}
    pathlib.Path(prefix + ".json").write_text(json.dumps(meta, indent=2) + "\n")
    return frames


def read_slices(prefix):
    """(meta dict, frames as a (frames, ny, nx) float32 array) of a PREFIX.f32 /
    PREFIX.json pair; a size that does not match the metadata is an error."""
    prefix = str(prefix)
    meta = json.loads(pathlib.Path(prefix + ".json").read_text())
    nx, ny, frames = meta["nx"], meta["ny"], meta["frames"]
    data = np.fromfile(prefix + ".f32", dtype=np.float32)
    if data.size != frames * nx * ny:
        raise ValueError(f"size mismatch: {data.size} floats, expected {frames * nx * ny}")
    return meta, data.reshape(frames, ny, nx)
