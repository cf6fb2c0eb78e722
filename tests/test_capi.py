"""CPU checks of the C ABI: the library loads, exports every entry point declared
in include/*.h, and rejects bad arguments before touching a device.  None of
these calls launches a kernel."""
from __future__ import annotations

import ctypes as C
import pathlib
import re

import pytest

import stencil_solver_b200 as sb

ROOT = pathlib.Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(sb200_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_loads_and_reports_version():
    assert sb.lib().sb200_version() >= 100


def test_every_declared_symbol_is_exported():
    L = sb.lib()
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, f"declared in include/ but not exported: {missing}"


def test_every_declared_symbol_has_a_binding():
    bound = set(sb.exported_symbols())
    unbound = [n for n in declared_symbols() if n not in bound]
    assert not unbound, f"no Python signature for {unbound}"


def test_null_grid_rejected():
    L = sb.lib()
    rc = L.sb200_launch_naive(8, 8, 8, 16, None, None)
    assert rc == sb.SB200_ERR_INVALID
    assert "grid" in sb.last_error()


def test_null_field_rejected():
    g = sb.Grid(32, 32, 32)
    with pytest.raises(sb.StencilError) as e:
        sb.launch_tiled(None, 16, 16, 32, g)
    assert e.value.status == sb.SB200_ERR_INVALID


def test_output_aliasing_current_field_rejected():
    g = sb.Grid(32, 32, 32)
    with pytest.raises(sb.StencilError, match="alias"):
        sb.launch_tiled(256, 512, 768, 256, g)
    with pytest.raises(sb.StencilError, match="alias"):
        sb.heat_step(256, 256, g, 1.0)


@pytest.mark.parametrize("bad", [dict(dx=0.0), dict(dy=-1.0), dict(dz=float("inf")),
                                 dict(dt=float("nan")), dict(nx=-4)])
def test_bad_grid_rejected(bad):
    kw = dict(nx=32, ny=32, nz=32, dx=10.0, dy=10.0, dz=10.0, dt=1e-3)
    kw.update(bad)
    with pytest.raises(sb.StencilError) as e:
        sb.launch_tiled(256, 512, 768, 1024, sb.Grid(**kw))
    assert e.value.status == sb.SB200_ERR_INVALID


def test_source_outside_grid_rejected():
    g = sb.Grid(32, 32, 32)
    with pytest.raises(sb.StencilError, match="source"):
        sb.wave_step(256, 512, 768, 1024, g, src_index=g.size, src_amp=1.0)


def test_grid_without_interior_is_a_noop():
    # The reference launchers launch no work when n <= 2R (stencil_naive.cu:63-64).
    g = sb.Grid(8, 8, 8)
    sb.launch_naive(256, 512, 768, 1024, g)
    sb.launch_tiled(256, 512, 768, 1024, g)
    sb.heat_step(256, 512, g, 1.0)


def test_override_validation():
    with pytest.raises(sb.StencilError):
        sb.set_pencil_override(7, 0, 1)
    with pytest.raises(sb.StencilError):
        sb.set_pencil_override(sb.KIND_WAVE_F32, 1000, 1)
    with pytest.raises(sb.StencilError):
        sb.set_pencil_override(sb.KIND_WAVE_F32, 0, 0)
    n = sb.lib().sb200_pencil_variant_count(sb.KIND_WAVE_F32)
    assert n >= 1 and len(sb.variant_names()) == n


def test_grid_struct_layout():
    # int64 x3 then float x4, naturally aligned: 40 bytes.
    assert C.sizeof(sb.sb200_grid) == 40


def test_tune_cache_load_skips_bad_lines(tmp_path):
    f = tmp_path / "tune.txt"
    f.write_text("0 1024 1024 1024 1 4 2.5 NVIDIA_B200\n"
                 "garbage line\n"
                 "0 64 64 64 999 1 1.0 NVIDIA_B200\n"   # variant out of range
                 "1 512 512 512 0 2 0.7 NVIDIA_B200\n")
    assert sb.tune_load(str(f)) == 2
    out = tmp_path / "out.txt"
    sb.tune_save(str(out))
    lines = out.read_text().split("\n")
    assert any(l.startswith("0 1024 1024 1024 1 4") for l in lines)
    assert any(l.startswith("1 512 512 512 0 2") for l in lines)


def test_two_step_argument_checks():
    """sb200_wave_step2_f32 wants five distinct fields: every aliasing of an output
    with an input, the two outputs with each other and p with p_prev is refused
    before any device work (the pointers are never dereferenced)."""
    g = sb.Grid(32, 32, 32)
    p, q, v, o1, o2 = 256, 512, 768, 1024, 1280
    for args in ((p, q, v, q, o2), (p, q, v, o1, p), (p, q, v, v, o2), (p, q, v, o1, o1),
                 (p, p, v, o1, o2)):
        with pytest.raises(sb.StencilError) as e:
            sb.wave_step2(*args, g)
        assert e.value.status == sb.SB200_ERR_INVALID
    with pytest.raises(sb.StencilError, match="NULL"):
        sb.wave_step2(p, q, None, o1, o2, g)
    with pytest.raises(sb.StencilError, match="source"):
        sb.wave_step2(p, q, v, o1, o2, g, src_index=g.size)
    sb.wave_step2(p, q, v, o1, o2, sb.Grid(8, 8, 8))  # no interior: nothing to do
    assert sb.variant_names(sb.KIND_WAVE2_F32)
