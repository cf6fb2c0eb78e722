"""B200-native stencil time-stepper (sm_100a) -- Python binding of the C ABI.

The product is the shared library ``lib/libstencil_b200.so`` (CUDA kernels + the
C ABI declared in ``include/stencil_b200.h``) together with the C++ drop-in API in
``include/stencil/``.  This module is a thin ctypes layer over the C ABI for
Python callers, the tests and the benchmark: device buffers are passed as raw
pointers or as CUDA tensors (anything with ``data_ptr()``), streams as raw
``cudaStream_t`` values or torch streams.

There is no CPU fallback: if the library is missing, loading fails loudly.
"""
from __future__ import annotations

import ctypes as C
import pathlib
from dataclasses import dataclass

PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libstencil_b200.so"

SB200_OK = 0
SB200_ERR_INVALID = -1
SB200_ERR_CUDA = -2
SB200_ERR_DEVICE = -3
SB200_ERR_UNSUPPORTED = -4
SB200_ERR_MONITOR = -5

KIND_WAVE_F32 = 0
KIND_HEAT_F32 = 1

R = 4  # stencil radius (8th order)


class StencilError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class sb200_grid(C.Structure):
    _fields_ = [("nx", C.c_int64), ("ny", C.c_int64), ("nz", C.c_int64),
                ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float), ("dt", C.c_float)]


@dataclass
class Grid:
    """Halo-inclusive grid (the reference's GridDims with an explicit dt)."""
    nx: int
    ny: int
    nz: int
    dx: float = 10.0
    dy: float = 10.0
    dz: float = 10.0
    dt: float = 1e-3

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)

    @property
    def size(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def interior(self) -> int:
        return max(self.nx - 2 * R, 0) * max(self.ny - 2 * R, 0) * max(self.nz - 2 * R, 0)

    def index(self, x: int, y: int, z: int) -> int:
        return (z * self.ny + y) * self.nx + x

    def c(self) -> sb200_grid:
        return sb200_grid(self.nx, self.ny, self.nz, self.dx, self.dy, self.dz, self.dt)


class sb200_run_config(C.Structure):
    _fields_ = [("grid", sb200_grid), ("physics", C.c_int), ("precision", C.c_int),
                ("exact", C.c_int), ("diffusivity", C.c_float), ("src_index", C.c_int64),
                ("src_freq", C.c_float), ("src_t0", C.c_float), ("graph_chunk", C.c_int),
                ("renorm_every", C.c_int), ("monitor_every", C.c_int),
                ("monitor_limit", C.c_float), ("f16_target", C.c_float)]


class sb200_shot(C.Structure):
    _fields_ = [("grid", sb200_grid), ("src_index", C.c_int64)]


class sb200_batch_config(C.Structure):
    _fields_ = [("precision", C.c_int), ("graph_chunk", C.c_int), ("max_steps", C.c_int64)]


class sb200_f16_scale(C.Structure):
    _fields_ = [("a", C.c_float), ("r", C.c_float)]


PHYSICS_WAVE, PHYSICS_HEAT = 0, 1
PRECISION_F32, PRECISION_F16 = 0, 1
KIND_WAVE_F16 = 2
KIND_WAVE2_F32 = 3  # wave_step2: two acoustic steps per sweep

_lib: C.CDLL | None = None

_SIGNATURES = {
    "sb200_version": ([], C.c_int),
    "sb200_last_error": ([], C.c_char_p),
    "sb200_device_error": ([C.c_int], C.c_int),
    "sb200_upload_fd_coefficients": ([], C.c_int),
    "sb200_launch_naive": ([C.c_void_p] * 4 + [C.POINTER(sb200_grid), C.c_void_p], C.c_int),
    "sb200_launch_tiled": ([C.c_void_p] * 4 + [C.POINTER(sb200_grid), C.c_void_p], C.c_int),
    "sb200_launch_slab": ([C.c_void_p] * 4 + [C.POINTER(sb200_grid), C.c_void_p], C.c_int),
    "sb200_wave_step_f32": ([C.c_void_p] * 4 + [C.POINTER(sb200_grid), C.c_int64, C.c_float,
                                                C.c_void_p], C.c_int),
    "sb200_wave_step_exact_f32": ([C.c_void_p] * 4 + [C.POINTER(sb200_grid), C.c_int64,
                                      C.c_float, C.c_void_p], C.c_int),
    "sb200_wave_step_dev_f32": ([C.c_void_p] * 4 + [C.POINTER(sb200_grid), C.c_int64,
                                    C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p],
                                   C.c_int),
    "sb200_wave_step2_f32": ([C.c_void_p] * 5 + [C.POINTER(sb200_grid), C.c_int64, C.c_float,
                                                 C.c_float, C.c_void_p], C.c_int),
    "sb200_wave_step2_dev_f32": ([C.c_void_p] * 5 + [C.POINTER(sb200_grid), C.c_int64,
                                     C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p],
                                    C.c_int),
    "sb200_set_device_int": ([C.c_void_p, C.c_int, C.c_void_p], C.c_int),
    "sb200_heat_step_exact_f32": ([C.c_void_p, C.c_void_p, C.POINTER(sb200_grid), C.c_float,
                                   C.c_void_p], C.c_int),
    "sb200_heat_step_f32": ([C.c_void_p, C.c_void_p, C.POINTER(sb200_grid), C.c_float,
                             C.c_void_p], C.c_int),
    "sb200_mlp_flags_compose": ([C.c_void_p, C.POINTER(sb200_grid), C.c_void_p, C.c_void_p,
                                 C.c_void_p], C.c_int),
    "sb200_wave_prepass_f32": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.POINTER(sb200_grid), C.c_float, C.c_void_p], C.c_int),
    "sb200_model_layered": ([C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_uint64, C.c_int,
                             C.c_float, C.c_float, C.c_float, C.c_float,
                             C.POINTER(C.c_float)], C.c_int),
    "sb200_ricker": ([C.c_double, C.c_double, C.c_double, C.c_int64, C.c_void_p], C.c_int),
    "sb200_tune": ([C.c_int, C.POINTER(sb200_grid)] + [C.c_void_p] * 4 +
                   [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float)],
                   C.c_int),
    "sb200_tune_save": ([C.c_char_p], C.c_int),
    "sb200_tune_load": ([C.c_char_p], C.c_int),
    "sb200_field_stats_scratch_len": ([C.POINTER(sb200_grid)], C.c_int64),
    "sb200_field_stats_f32": ([C.c_void_p, C.POINTER(sb200_grid), C.c_void_p, C.c_void_p,
                               C.c_int64, C.c_void_p], C.c_int),
    "sb200_field_stats_f16": ([C.c_void_p, C.POINTER(sb200_grid), C.c_float, C.c_void_p,
                               C.c_void_p, C.c_int64, C.c_void_p], C.c_int),
    "sb200_field_stats_f32_noalloc": ([C.c_void_p, C.POINTER(sb200_grid), C.c_void_p, C.c_void_p],
                                      C.c_int),
    "sb200_f16_pack": ([C.c_void_p, C.c_void_p, C.c_int64, C.c_float, C.c_void_p], C.c_int),
    "sb200_f16_unpack": ([C.c_void_p, C.c_void_p, C.c_int64, C.c_float, C.c_void_p], C.c_int),
    "sb200_k_field_bf16": ([C.c_void_p, C.c_void_p, C.POINTER(sb200_grid), C.c_void_p], C.c_int),
    "sb200_wave_step_f16": ([C.c_void_p] * 3 + [C.POINTER(sb200_grid), C.c_int64, C.c_float,
                            C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p],
                           C.c_int),
    "sb200_f16_renorm": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_float,
                          C.c_void_p], C.c_int),
    "sb200_run_config_init": ([C.POINTER(sb200_run_config), C.POINTER(sb200_grid)], None),
    "sb200_run_create": ([C.POINTER(sb200_run_config), C.POINTER(C.c_void_p)], C.c_int),
    "sb200_run_destroy": ([C.c_void_p], C.c_int),
    "sb200_run_set_fields": ([C.c_void_p] * 4, C.c_int),
    "sb200_run_set_wavelet": ([C.c_void_p, C.c_void_p, C.c_int64], C.c_int),
    "sb200_run_steps": ([C.c_void_p, C.c_int64], C.c_int),
    "sb200_run_synchronize": ([C.c_void_p], C.c_int),
    "sb200_run_get_field": ([C.c_void_p, C.c_void_p], C.c_int),
    "sb200_run_get_plane": ([C.c_void_p, C.c_int64, C.c_void_p], C.c_int),
    "sb200_run_get_trace": ([C.c_void_p, C.c_void_p, C.c_int64], C.c_int),
    "sb200_run_stats": ([C.c_void_p, C.c_void_p], C.c_int),
    "sb200_run_steps_done": ([C.c_void_p], C.c_int64),
    "sb200_run_stream": ([C.c_void_p], C.c_void_p),
    "sb200_batch_config_init": ([C.POINTER(sb200_batch_config)], None),
    "sb200_batch_create": ([C.POINTER(sb200_shot), C.c_int, C.POINTER(sb200_batch_config),
                            C.POINTER(C.c_void_p)], C.c_int),
    "sb200_batch_destroy": ([C.c_void_p], C.c_int),
    "sb200_batch_set_fields": ([C.c_void_p, C.c_int] + [C.c_void_p] * 3, C.c_int),
    "sb200_batch_set_wavelet": ([C.c_void_p, C.c_int, C.c_void_p, C.c_int64], C.c_int),
    "sb200_batch_steps": ([C.c_void_p, C.c_int64], C.c_int),
    "sb200_batch_synchronize": ([C.c_void_p], C.c_int),
    "sb200_batch_get_field": ([C.c_void_p, C.c_int, C.c_void_p], C.c_int),
    "sb200_batch_get_trace": ([C.c_void_p, C.c_int, C.c_void_p, C.c_int64], C.c_int),
    "sb200_batch_tune": ([C.c_void_p, C.c_int], C.c_int),
    "sb200_batch_set_monitor_limit": ([C.c_void_p, C.c_float], C.c_int),
    "sb200_batch_monitor_flags": ([C.c_void_p, C.c_void_p], C.c_int),
    "sb200_batch_set_choice": ([C.c_void_p, C.c_int, C.c_int], C.c_int),
    "sb200_batch_choice": ([C.c_void_p] + [C.POINTER(C.c_int)] * 4, C.c_int),
    "sb200_batch_steps_done": ([C.c_void_p], C.c_int64),
    "sb200_batch_stream": ([C.c_void_p], C.c_void_p),
    "sb200_batch_variant_count": ([], C.c_int),
    "sb200_batch_variant_count_f16": ([], C.c_int),
    "sb200_batch_variant_name_f16": ([C.c_int], C.c_char_p),
    "sb200_batch_variant_name": ([C.c_int], C.c_char_p),
    "sb200_mlp_create": ([C.c_uint64, C.POINTER(C.c_void_p)], C.c_int),
    "sb200_mlp_destroy": ([C.c_void_p], C.c_int),
    "sb200_mlp_get_params": ([C.c_void_p, C.c_void_p], C.c_int),
    "sb200_mlp_set_params": ([C.c_void_p, C.c_void_p], C.c_int),
    "sb200_mlp_set_output_scale": ([C.c_void_p, C.c_float], C.c_int),
    "sb200_mlp_set_kernel": ([C.c_void_p, C.c_int], C.c_int),
    "sb200_mlp_output_scale": ([C.c_void_p], C.c_float),
    "sb200_mlp_forward": ([C.c_void_p] * 3 + [C.c_int64, C.c_void_p], C.c_int),
    "sb200_mlp_gradients": ([C.c_void_p] * 3 + [C.c_int64, C.c_void_p, C.c_void_p], C.c_int),
    "sb200_mlp_train_step": ([C.c_void_p] * 3 + [C.c_int64, C.c_float, C.c_void_p, C.c_void_p],
                             C.c_int),
    "sb200_mlp_correct": ([C.c_void_p] * 4 + [C.POINTER(sb200_grid), C.c_void_p], C.c_int),
    "sb200_mlp_learned_step": ([C.c_void_p] * 4 + [C.POINTER(sb200_grid), C.c_void_p], C.c_int),
    "sb200_mlp_flags_bytes": ([C.c_void_p, C.POINTER(sb200_grid)], C.c_int64),
    "sb200_mlp_learned_step_flags": ([C.c_void_p] * 4 + [C.POINTER(sb200_grid)] + [C.c_void_p] * 4,
                                     C.c_int),
    "sb200_mlp_set_min_scale": ([C.c_void_p, C.c_float], C.c_int),
    "sb200_mlp_min_scale": ([C.c_void_p], C.c_float),
    "sb200_mlp_samples": ([C.c_void_p] * 4 + [C.POINTER(sb200_grid), C.c_void_p, C.c_int64,
                                               C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "sb200_add_box": ([C.c_void_p, C.POINTER(sb200_grid)] + [C.c_int] * 6 +
                      [C.c_void_p, C.c_float, C.c_void_p], C.c_int),
    "sb200_smooth3": ([C.c_void_p, C.c_void_p, C.POINTER(sb200_grid), C.c_float, C.c_void_p],
                      C.c_int),
    "sb200_restrict2": ([C.c_void_p, C.POINTER(sb200_grid), C.c_void_p, C.POINTER(sb200_grid),
                         C.c_int, C.c_void_p], C.c_int),
    "sb200_pencil_variant_count": ([C.c_int], C.c_int),
    "sb200_pencil_variant_name": ([C.c_int, C.c_int], C.c_char_p),
    "sb200_set_pencil_override": ([C.c_int, C.c_int, C.c_int], C.c_int),
    "sb200_pencil_choice": ([C.c_int, C.POINTER(sb200_grid), C.POINTER(C.c_int),
                             C.POINTER(C.c_int)], C.c_int),
}


def lib() -> C.CDLL:
    """Loads libstencil_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; "
                "g.build()'` (requires nvcc); there is no CPU fallback")
        L = C.CDLL(str(LIB_PATH))
        for name, (args, res) in _SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def exported_symbols():
    return sorted(_SIGNATURES)


def last_error() -> str:
    s = lib().sb200_last_error()
    return s.decode() if s else ""


def _check(status: int) -> int:
    if status < 0:
        raise StencilError(status, last_error())
    return status


def _ptr(x) -> int | None:
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    raise TypeError(f"expected a device pointer or tensor, got {type(x)!r}")


def _stream(s) -> int | None:
    if s is None:
        return None
    if isinstance(s, int):
        return s
    if hasattr(s, "cuda_stream"):
        return s.cuda_stream
    raise TypeError(f"expected a cudaStream_t or torch stream, got {type(s)!r}")


def _g(grid: Grid):
    return C.byref(grid.c())


def upload_fd_coefficients() -> None:
    _check(lib().sb200_upload_fd_coefficients())


def launch_naive(p_cur, p_prev, vel2, p_next, grid: Grid, stream=None) -> None:
    _check(lib().sb200_launch_naive(_ptr(p_cur), _ptr(p_prev), _ptr(vel2), _ptr(p_next),
                                    _g(grid), _stream(stream)))


def launch_tiled(p_cur, p_prev, vel2, p_next, grid: Grid, stream=None) -> None:
    _check(lib().sb200_launch_tiled(_ptr(p_cur), _ptr(p_prev), _ptr(vel2), _ptr(p_next),
                                    _g(grid), _stream(stream)))


def launch_slab(p_cur, p_prev, vel2, p_next, grid: Grid, stream=None) -> None:
    _check(lib().sb200_launch_slab(_ptr(p_cur), _ptr(p_prev), _ptr(vel2), _ptr(p_next),
                                   _g(grid), _stream(stream)))


def wave_step(p, p_prev, vel2, p_next, grid: Grid, src_index: int = -1, src_amp: float = 0.0,
              stream=None) -> None:
    _check(lib().sb200_wave_step_f32(_ptr(p), _ptr(p_prev), _ptr(vel2), _ptr(p_next), _g(grid),
                                     src_index, src_amp, _stream(stream)))


def wave_step_exact(p, p_prev, vel2, p_next, grid: Grid, src_index: int = -1,
                    src_amp: float = 0.0, stream=None) -> None:
    _check(lib().sb200_wave_step_exact_f32(_ptr(p), _ptr(p_prev), _ptr(vel2), _ptr(p_next),
                                           _g(grid), src_index, src_amp, _stream(stream)))


def heat_step(u, u_next, grid: Grid, alpha: float, stream=None) -> None:
    _check(lib().sb200_heat_step_f32(_ptr(u), _ptr(u_next), _g(grid), alpha, _stream(stream)))


def model_layered(nx: int, ny: int, nz: int, seed: int, n_layers: int = 8,
                  v_top: float = 1500.0, v_bottom: float = 4500.0, perturbation: float = 0.05,
                  corr_cells: float = 20.0, out=None):
    """Seeded layered v^2 model as a (nz, ny, nx) float32 numpy array; returns (vel2, v_max)."""
    import numpy as np

    if out is None:
        out = np.empty((nz, ny, nx), np.float32)
    vmax = C.c_float()
    _check(lib().sb200_model_layered(out.ctypes.data, nx, ny, nz, seed, n_layers, v_top,
                                     v_bottom, perturbation, corr_cells, C.byref(vmax)))
    return out, float(vmax.value)


def ricker(freq: float, t0: float, dt: float, n_steps: int):
    import numpy as np

    out = np.empty(n_steps, np.float32)
    _check(lib().sb200_ricker(freq, t0, dt, n_steps, out.ctypes.data))
    return out


def wave_prepass(p, p_prev, vel2, r, grid: Grid, beta: float = 1.0 / 16.0, stream=None) -> None:
    """r = p + beta dt^2 v^2 lap p; p_prev += 2 beta dt^2 v^2 lap p (sb200_wave_prepass_f32):
    a plain step of (r, p_prev) then carries the beta dt^4 L^2 p term."""
    _check(lib().sb200_wave_prepass_f32(_ptr(p), _ptr(p_prev), _ptr(vel2), _ptr(r), _g(grid),
                                        C.c_float(beta), _stream(stream)))


def heat_step_exact(u, u_next, grid: Grid, alpha: float, stream=None) -> None:
    _check(lib().sb200_heat_step_exact_f32(_ptr(u), _ptr(u_next), _g(grid), alpha,
                                           _stream(stream)))


def wave_step_dev(p, p_prev, vel2, p_next, grid: Grid, src_index: int, wavelet, step,
                  step_offset: int = 0, exact: bool = False, stream=None) -> None:
    _check(lib().sb200_wave_step_dev_f32(_ptr(p), _ptr(p_prev), _ptr(vel2), _ptr(p_next),
                                         _g(grid), src_index, _ptr(wavelet), _ptr(step),
                                         step_offset, 1 if exact else 0, _stream(stream)))


def wave_step2(p, p_prev, vel2, p_next, p_next2, grid: Grid, src_index: int = -1,
               src_amp0: float = 0.0, src_amp1: float = 0.0, stream=None) -> None:
    """Two acoustic steps in one sweep: p_next = step(p, p_prev) with sample
    src_amp0, p_next2 = step(p_next, p) with src_amp1 (five distinct buffers)."""
    _check(lib().sb200_wave_step2_f32(_ptr(p), _ptr(p_prev), _ptr(vel2), _ptr(p_next),
                                      _ptr(p_next2), _g(grid), src_index, src_amp0, src_amp1,
                                      _stream(stream)))


def wave_step2_dev(p, p_prev, vel2, p_next, p_next2, grid: Grid, src_index: int, wavelet, step,
                   step_offset: int = 0, trace=None, stream=None) -> None:
    _check(lib().sb200_wave_step2_dev_f32(_ptr(p), _ptr(p_prev), _ptr(vel2), _ptr(p_next),
                                          _ptr(p_next2), _g(grid), src_index, _ptr(wavelet),
                                          _ptr(step), step_offset, _ptr(trace),
                                          _stream(stream)))


def set_device_int(dst, value: int, stream=None) -> None:
    _check(lib().sb200_set_device_int(_ptr(dst), value, _stream(stream)))


def field_stats_scratch_len(grid: Grid) -> int:
    return _check(lib().sb200_field_stats_scratch_len(_g(grid)))


def field_stats(field, grid: Grid, out3, scratch, scale: float = 1.0, stream=None) -> None:
    """Enqueues the FP64 interior statistics {sum f^2, max|f|, non-finite count} of an
    FP32 or FP16 (by dtype; values stored times `scale`) field into the 3-double out3.
    scratch is a float64 device tensor of at least field_stats_scratch_len(grid)."""
    n = scratch.numel()
    if str(field.dtype).endswith("float16"):
        _check(lib().sb200_field_stats_f16(_ptr(field), _g(grid), scale, _ptr(out3),
                                           _ptr(scratch), n, _stream(stream)))
    else:
        _check(lib().sb200_field_stats_f32(_ptr(field), _g(grid), _ptr(out3), _ptr(scratch), n,
                                           _stream(stream)))


def field_stats_noalloc(field, grid: Grid, out3, stream=None) -> None:
    """field_stats of an FP32 field with the library's static device scratch:
    allocates nothing.  Calls that overlap on the device share that scratch."""
    _check(lib().sb200_field_stats_f32_noalloc(_ptr(field), _g(grid), _ptr(out3),
                                               _stream(stream)))


def f16_pack(src, dst, n: int, scale: float, stream=None) -> None:
    _check(lib().sb200_f16_pack(_ptr(src), _ptr(dst), n, scale, _stream(stream)))


def f16_unpack(src, dst, n: int, scale: float, stream=None) -> None:
    _check(lib().sb200_f16_unpack(_ptr(src), _ptr(dst), n, scale, _stream(stream)))


def k_field_bf16(vel2, k, grid: Grid, stream=None) -> None:
    _check(lib().sb200_k_field_bf16(_ptr(vel2), _ptr(k), _g(grid), _stream(stream)))


def wave_step_f16(p, p_prev_next, k, grid: Grid, scale, phase: int = 0, src_index: int = -1,
                  src_amp: float = 0.0, wavelet=None, step=None, step_offset: int = 0,
                  stream=None) -> None:
    _check(lib().sb200_wave_step_f16(_ptr(p), _ptr(p_prev_next), _ptr(k), _g(grid), src_index,
                                     src_amp, _ptr(wavelet), _ptr(step), step_offset, _ptr(scale),
                                     phase, _stream(stream)))


def f16_renorm(stats3, scale, bound_host: float, target: float = 4096.0, bound=None, step=None,
               stream=None) -> None:
    _check(lib().sb200_f16_renorm(_ptr(stats3), _ptr(scale), _ptr(bound), _ptr(step), bound_host,
                                  target, _stream(stream)))


class Run:
    """A whole simulation behind the C-ABI run handle (sb200_run_*): fields in from
    host memory, steps on the device (CUDA-graph chunks), results back to host memory.

    Keyword options map onto sb200_run_config (physics, precision, exact, diffusivity,
    src_index, src_freq, src_t0, graph_chunk, renorm_every, monitor_every,
    monitor_limit, f16_target)."""

    def __init__(self, grid: Grid, **opts):
        cfg = sb200_run_config()
        lib().sb200_run_config_init(C.byref(cfg), _g(grid))
        for k, v in opts.items():
            if not hasattr(cfg, k):
                raise TypeError(f"unknown run option {k!r}")
            setattr(cfg, k, v)
        h = C.c_void_p()
        _check(lib().sb200_run_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._destroy = lib().sb200_run_destroy  # still callable at interpreter exit
        self.grid = grid

    def close(self):
        if getattr(self, "_h", None):
            self._destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def _host(a):
        import numpy as np

        if a is None:
            return None
        if hasattr(a, "data_ptr"):  # a host tensor (pinned or not)
            return a.data_ptr()
        a = np.ascontiguousarray(a, dtype=np.float32)
        return a.ctypes.data, a

    def set_fields(self, p, p_prev=None, vel2=None) -> None:
        keep = []
        ptrs = []
        for x in (p, p_prev, vel2):
            h = self._host(x)
            if isinstance(h, tuple):
                keep.append(h[1])
                h = h[0]
            ptrs.append(h)
        _check(lib().sb200_run_set_fields(self._h, *ptrs))

    def set_wavelet(self, w) -> None:
        import numpy as np

        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(lib().sb200_run_set_wavelet(self._h, w.ctypes.data, w.size))

    def steps(self, n: int) -> None:
        _check(lib().sb200_run_steps(self._h, n))

    def synchronize(self) -> None:
        _check(lib().sb200_run_synchronize(self._h))

    def field(self, out=None):
        import numpy as np

        if out is None:
            out = np.empty(self.grid.shape, np.float32)
        ptr = out.data_ptr() if hasattr(out, "data_ptr") else out.ctypes.data
        _check(lib().sb200_run_get_field(self._h, ptr))
        return out

    def plane(self, z: int, out=None):
        """XY plane z of the current field, (ny, nx) float32, physical units."""
        import numpy as np

        g = self.grid
        if out is None:
            out = np.empty((g.ny, g.nx), np.float32)
        _check(lib().sb200_run_get_plane(self._h, int(z), out.ctypes.data))
        return out

    def trace(self, n: int):
        import numpy as np

        out = np.empty(n, np.float32)
        _check(lib().sb200_run_get_trace(self._h, out.ctypes.data, n))
        return out

    def stats(self):
        import numpy as np

        out = np.zeros(3, np.float64)
        _check(lib().sb200_run_stats(self._h, out.ctypes.data))
        return out

    @property
    def steps_done(self) -> int:
        return lib().sb200_run_steps_done(self._h)

    @property
    def stream(self) -> int:
        return lib().sb200_run_stream(self._h) or 0


def device_error(clear: bool = True) -> int:
    return _check(lib().sb200_device_error(1 if clear else 0))


def variant_names(kind: int = KIND_WAVE_F32):
    n = _check(lib().sb200_pencil_variant_count(kind))
    return [lib().sb200_pencil_variant_name(kind, i).decode() for i in range(n)]


def tune(kind: int, grid: Grid, field, prev, vel2, scratch, reps: int = 3):
    """Autotunes the pencil tile / z split for kind on grid; returns (variant, zchunks, ms)."""
    v, z, ms = C.c_int(), C.c_int(), C.c_float()
    _check(lib().sb200_tune(kind, _g(grid), _ptr(field), _ptr(prev), _ptr(vel2), _ptr(scratch),
                            reps, C.byref(v), C.byref(z), C.byref(ms)))
    return v.value, z.value, ms.value


def tune_save(path: str) -> None:
    _check(lib().sb200_tune_save(str(path).encode()))


def tune_load(path: str) -> int:
    return _check(lib().sb200_tune_load(str(path).encode()))


def set_pencil_override(kind: int, variant: int, zchunks: int = 1) -> None:
    _check(lib().sb200_set_pencil_override(kind, variant, zchunks))


def pencil_choice(kind: int, grid: Grid):
    v, z = C.c_int(), C.c_int()
    _check(lib().sb200_pencil_choice(kind, _g(grid), C.byref(v), C.byref(z)))
    return v.value, z.value


class Batch:
    """Independent acoustic shots of uneven sizes advanced together by one
    persistent launch per step (C-ABI handle sb200_batch_*).  shots is a list of
    (Grid, src_index) pairs; max_steps bounds the run (source and trace tables).
    precision PRECISION_F16 stores p / p_prev in FP16 at per-shot power-of-two
    scales (renormalised every 50 steps from FP64 statistics) and K in BF16
    (every nx a multiple of 8); fields and traces cross the boundary in FP32."""

    def __init__(self, shots, max_steps: int, graph_chunk: int = 100,
                 precision: int = PRECISION_F32):
        arr = (sb200_shot * len(shots))()
        for i, (g, src) in enumerate(shots):
            arr[i].grid = g.c()
            arr[i].src_index = -1 if src is None else int(src)
        cfg = sb200_batch_config()
        lib().sb200_batch_config_init(C.byref(cfg))
        cfg.graph_chunk = graph_chunk
        cfg.max_steps = max_steps
        cfg.precision = precision
        h = C.c_void_p()
        _check(lib().sb200_batch_create(arr, len(shots), C.byref(cfg), C.byref(h)))
        self._h = h
        self._destroy = lib().sb200_batch_destroy  # still callable at interpreter exit
        self.grids = [g for g, _ in shots]
        self.precision = precision

    def close(self):
        if getattr(self, "_h", None):
            self._destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_fields(self, shot: int, p, p_prev=None, vel2=None) -> None:
        import numpy as np

        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float32)
                for a in (p, p_prev, vel2)]
        ptrs = [None if a is None else a.ctypes.data for a in arrs]
        _check(lib().sb200_batch_set_fields(self._h, shot, *ptrs))

    def set_wavelet(self, shot: int, w) -> None:
        import numpy as np

        w = np.ascontiguousarray(w, dtype=np.float32)
        _check(lib().sb200_batch_set_wavelet(self._h, shot, w.ctypes.data, w.size))

    def steps(self, n: int) -> None:
        _check(lib().sb200_batch_steps(self._h, n))

    def synchronize(self) -> None:
        _check(lib().sb200_batch_synchronize(self._h))

    def set_monitor_limit(self, limit: float) -> None:
        """Largest |p| the FP32 stability monitor accepts (default 1e30)."""
        _check(lib().sb200_batch_set_monitor_limit(self._h, float(limit)))

    def monitor_flags(self):
        """Per-shot monitor flags (1: non-finite value or |p| above the limit)."""
        import numpy as np

        out = np.zeros(len(self.grids), np.int32)
        _check(lib().sb200_batch_monitor_flags(self._h, out.ctypes.data))
        return out

    def field(self, shot: int):
        import numpy as np

        out = np.empty(self.grids[shot].shape, np.float32)
        _check(lib().sb200_batch_get_field(self._h, shot, out.ctypes.data))
        return out

    def trace(self, shot: int, n: int):
        import numpy as np

        out = np.empty(n, np.float32)
        _check(lib().sb200_batch_get_trace(self._h, shot, out.ctypes.data, n))
        return out

    def tune(self, reps: int = 3) -> None:
        _check(lib().sb200_batch_tune(self._h, reps))

    def set_choice(self, variant: int, zlen: int) -> None:
        _check(lib().sb200_batch_set_choice(self._h, variant, zlen))

    def choice(self) -> dict:
        v, z, n, c = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        _check(lib().sb200_batch_choice(self._h, C.byref(v), C.byref(z), C.byref(n), C.byref(c)))
        name = (lib().sb200_batch_variant_name_f16 if self.precision == PRECISION_F16
                else lib().sb200_batch_variant_name)(v.value)
        return {"variant": v.value, "zlen": z.value, "items": n.value, "ctas": c.value,
                "name": name.decode()}

    @property
    def steps_done(self) -> int:
        return _check(lib().sb200_batch_steps_done(self._h))

    @property
    def stream(self) -> int:
        return lib().sb200_batch_stream(self._h)


MLP_NPARAM = 2145
MLP_FEATURES = 32


class Mlp:
    """The learned-correction network (sb200_mlp_*): FP32 parameters on the device,
    BF16 tensor-core forward / backward, Adam.  Feature rows are int16 / uint16
    CUDA tensors of shape (n, 32) holding BF16 bit patterns."""

    def __init__(self, seed: int = 0):
        h = C.c_void_p()
        _check(lib().sb200_mlp_create(seed, C.byref(h)))
        self._h = h
        self._destroy = lib().sb200_mlp_destroy  # still callable at interpreter exit

    def close(self):
        if getattr(self, "_h", None):
            self._destroy(self._h)
            self._h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    def params(self):
        import numpy as np

        out = np.empty(MLP_NPARAM, np.float32)
        _check(lib().sb200_mlp_get_params(self._h, out.ctypes.data))
        return out

    def set_params(self, w) -> None:
        import numpy as np

        w = np.ascontiguousarray(w, np.float32)
        if w.size != MLP_NPARAM:
            raise ValueError(f"expected {MLP_NPARAM} parameters")
        _check(lib().sb200_mlp_set_params(self._h, w.ctypes.data))

    @property
    def output_scale(self) -> float:
        return float(lib().sb200_mlp_output_scale(self._h))

    @output_scale.setter
    def output_scale(self, c: float) -> None:
        _check(lib().sb200_mlp_set_output_scale(self._h, c))

    @property
    def min_scale(self) -> float:
        """Correction floor: points whose star's largest magnitude is below it get
        no correction (0, the default: every point with a nonzero star)."""
        return float(lib().sb200_mlp_min_scale(self._h))

    @min_scale.setter
    def min_scale(self, floor: float) -> None:
        _check(lib().sb200_mlp_set_min_scale(self._h, floor))

    def set_kernel(self, kernel: str) -> None:
        """Correction kernel: "tcgen05" (default) or "mma"."""
        _check(lib().sb200_mlp_set_kernel(self._h, {"tcgen05": 0, "mma": 1}[kernel]))

    def forward(self, X, y, n=None, stream=None) -> None:
        n = X.shape[0] if n is None else n
        _check(lib().sb200_mlp_forward(self._h, _ptr(X), _ptr(y), n, _stream(stream)))

    def gradients(self, X, t, grad, n=None, stream=None) -> None:
        n = X.shape[0] if n is None else n
        _check(lib().sb200_mlp_gradients(self._h, _ptr(X), _ptr(t), n, _ptr(grad),
                                          _stream(stream)))

    def train_step(self, X, t, lr: float, loss=None, n=None, stream=None) -> None:
        n = X.shape[0] if n is None else n
        _check(lib().sb200_mlp_train_step(self._h, _ptr(X), _ptr(t), n, lr, _ptr(loss),
                                           _stream(stream)))

    def correct(self, p, vel2, p_next, grid: Grid, stream=None) -> None:
        _check(lib().sb200_mlp_correct(self._h, _ptr(p), _ptr(vel2), _ptr(p_next), _g(grid),
                                        _stream(stream)))

    def learned_step(self, p, p_prev_next, vel2, grid: Grid, stream=None, flags=None,
                     box=None) -> None:
        """p_prev_next <- acoustic step of p + the learned correction, in one fused
        launch (no source term); the same bits as wave_step then correct.

        flags = (flags_in, flags_out): uint8 device tensors of flags_bytes(grid)
        bytes (flags_in None: every chunk active); chunks whose neighbourhood holds
        no flagged chunk skip the network.  box = (x0, x1, y0, y1, z0, z1) cells
        that count as flagged (a source added to p after its flags were written)."""
        if flags is None:
            _check(lib().sb200_mlp_learned_step(self._h, _ptr(p), _ptr(p_prev_next), _ptr(vel2),
                                                 _g(grid), _stream(stream)))
            return
        fin, fout = flags
        bx = None if box is None else (C.c_int64 * 6)(*[int(v) for v in box])
        _check(lib().sb200_mlp_learned_step_flags(
            self._h, _ptr(p), _ptr(p_prev_next), _ptr(vel2), _g(grid),
            None if fin is None else _ptr(fin), None if fout is None else _ptr(fout),
            None if bx is None else C.cast(bx, C.c_void_p), _stream(stream)))

    def flags_compose(self, grid: Grid, flags_p, flags_r, stream=None) -> None:
        """flags_r = activity flags of wave_prepass's r from those of p."""
        _check(lib().sb200_mlp_flags_compose(self._h, _g(grid), _ptr(flags_p), _ptr(flags_r),
                                             _stream(stream)))

    def flags_bytes(self, grid: Grid) -> int:
        """Bytes of the activity flags of learned_step on `grid`."""
        n = lib().sb200_mlp_flags_bytes(self._h, _g(grid))
        if n < 0:
            _check(int(n))
        return int(n)


def mlp_samples(p, vel2, p_true, p_plain, grid: Grid, cells, X, t, stream=None) -> None:
    _check(lib().sb200_mlp_samples(_ptr(p), _ptr(vel2), _ptr(p_true), _ptr(p_plain), _g(grid),
                                   _ptr(cells), cells.numel(), _ptr(X), _ptr(t),
                                   _stream(stream)))


def restrict2(fine, fine_grid: Grid, coarse, coarse_grid: Grid, offset: int = -4,
              stream=None) -> None:
    _check(lib().sb200_restrict2(_ptr(fine), _g(fine_grid), _ptr(coarse), _g(coarse_grid),
                                 offset, _stream(stream)))


def add_box(field, grid: Grid, origin, dims, pattern, scale: float, stream=None) -> None:
    """field[box] += scale * pattern, box at origin (x, y, z) of dims (bx, by, bz)."""
    _check(lib().sb200_add_box(_ptr(field), _g(grid), *origin, *dims, _ptr(pattern), scale,
                               _stream(stream)))


def smooth3(field, tmp, grid: Grid, sigma_cells: float, stream=None) -> None:
    """In-place separable Gaussian smoothing of a device field (tmp: same size)."""
    _check(lib().sb200_smooth3(_ptr(field), _ptr(tmp), _g(grid), sigma_cells, _stream(stream)))
