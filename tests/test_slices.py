"""The slice writer's file format (the reference's src/main_slice.cpp:15-19,
106-152), driven by a stand-in run on the host."""
from __future__ import annotations

import json

import numpy as np
import pytest

import stencil_solver_b200 as sb
from stencil_solver_b200.slices import META_KEYS, read_slices, write_slices


class FakeRun:
    """A field that is the step count everywhere plus x + 1000 y + 1e6 z."""

    def __init__(self, nx, ny, nz):
        self.grid = sb.Grid(nx, ny, nz, 10.0, 10.0, 10.0, 1e-3)
        self.step = 0
        self.calls = []

    def steps(self, n):
        self.calls.append(n)
        self.step += n

    def plane(self, z, out):
        ny, nx = out.shape
        y, x = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
        out[...] = self.step + x + 1000.0 * y + 1e6 * z
        return out


@pytest.mark.parametrize("steps,every,frames", [(20, 5, 5), (22, 5, 5), (3, 5, 1), (0, 4, 1),
                                                (7, 1, 8)])
def test_frames_and_metadata(tmp_path, steps, every, frames):
    run = FakeRun(12, 10, 9)
    prefix = tmp_path / "wave"
    n = write_slices(run, prefix, steps, every, velocity=2000.0)
    assert n == frames and run.step == steps and sum(run.calls) == steps
    meta, data = read_slices(prefix)
    assert tuple(meta) == META_KEYS
    assert meta["frames"] == frames and meta["every"] == every and meta["steps"] == steps
    assert (meta["nx"], meta["ny"], meta["nz"], meta["plane"]) == (12, 10, 9, "xy")
    assert meta["plane_index"] == 4 and meta["dtype"] == "float32"
    assert meta["velocity"] == 2000.0 and meta["physics"] == "wave"
    assert data.shape == (frames, 10, 12)
    # frame k is the state after k * every steps, x fastest
    for k in range(frames):
        assert data[k, 0, 0] == k * every + 4e6
        assert data[k, 0, 1] - data[k, 0, 0] == 1.0
        assert data[k, 1, 0] - data[k, 0, 0] == 1000.0
    assert (prefix.with_suffix(".f32")).stat().st_size == frames * 12 * 10 * 4


def test_plane_choice_and_errors(tmp_path):
    run = FakeRun(8, 8, 8)
    write_slices(run, tmp_path / "a", 2, 1, plane_index=0)
    meta, data = read_slices(tmp_path / "a")
    assert meta["plane_index"] == 0 and data[0, 0, 0] == 0.0
    for kw in ({"every": 0}, {"plane_index": 8}, {"plane_index": -1}):
        with pytest.raises(ValueError):
            write_slices(FakeRun(8, 8, 8), tmp_path / "b", 2, **{"every": 1, **kw})
    with pytest.raises(ValueError):
        write_slices(FakeRun(8, 8, 8), tmp_path / "c", -1)


def test_size_mismatch_is_an_error(tmp_path):
    run = FakeRun(8, 8, 8)
    write_slices(run, tmp_path / "w", 4, 2)
    meta = json.loads((tmp_path / "w.json").read_text())
    meta["frames"] += 1
    (tmp_path / "w.json").write_text(json.dumps(meta))
    with pytest.raises(ValueError):
        read_slices(tmp_path / "w")
