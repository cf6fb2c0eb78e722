"""ctypes bindings for the oracle (TEST INFRASTRUCTURE ONLY).

The oracle is the checker for the CUDA path.  Only tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline / reference legs may import this package.  The
product package (stencil_solver_b200) never imports it.

  liboracle.so          C restatement of the reference CPU path
                        (src/kernels/stencil_naive.cu:136-170, FP32 and FP64)
  _ref/libstencil_ref_* the reference's own CPU path compiled from its sources
"""
from __future__ import annotations

import ctypes as C
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i64 = C.c_int64

_lib = None
_ref = {}


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            from . import build as _b  # noqa: WPS433 -- build on first use (CPU only)
            _b.build_oracle()
        L = C.CDLL(str(path))
        for T, P, sfx in ((C.c_float, _f32p, "f32"), (C.c_double, _f64p, "f64")):
            f = getattr(L, f"oracle_wave_step_{sfx}")
            f.argtypes = [P, P, P, P, _i64, _i64, _i64, T, T, T, T]
            f.restype = None
            f = getattr(L, f"oracle_heat_step_{sfx}")
            f.argtypes = [P, P, _i64, _i64, _i64, T, T, T, T, T]
            f.restype = None
            f = getattr(L, f"oracle_wave_run_{sfx}")
            f.argtypes = [P, P, P, P, _i64, _i64, _i64, T, T, T, T, _i64, _i64,
                          C.c_void_p, C.c_void_p]
            f.restype = None
        L.oracle_ricker.argtypes = [C.c_double, C.c_double, C.c_double, _i64, _f64p]
        L.oracle_ricker.restype = None
        L.oracle_fd_coefficients.argtypes = [_f64p]
        L.oracle_fd_coefficients.restype = None
        _u16p = np.ctypeslib.ndpointer(dtype=np.uint16, flags="C_CONTIGUOUS")
        L.oracle_wave_step_f16.argtypes = [_u16p, _u16p, _u16p, _u16p, _i64, _i64, _i64, C.c_float,
                                           C.c_float, C.c_float, C.c_float, C.c_float, _i64,
                                           C.c_float, C.c_float]
        L.oracle_wave_step_f16.restype = None
        L.oracle_f32_to_f16.argtypes = [C.c_float]
        L.oracle_f32_to_f16.restype = C.c_uint16
        L.oracle_f16_to_f32.argtypes = [C.c_uint16]
        L.oracle_f16_to_f32.restype = C.c_float
        L.oracle_f32_to_bf16.argtypes = [C.c_float]
        L.oracle_f32_to_bf16.restype = C.c_uint16
        L.oracle_bf16_to_f32.argtypes = [C.c_uint16]
        L.oracle_bf16_to_f32.restype = C.c_float
        L.oracle_mlp_nparam.restype = C.c_int
        L.oracle_mlp_features.argtypes = [_f32p, _f32p, _i64, _i64, _i64, C.c_float, _u16p]
        L.oracle_mlp_features.restype = C.c_float
        L.oracle_mlp_forward.argtypes = [_f32p, _u16p, _i64, C.c_int, _f64p]
        L.oracle_mlp_forward.restype = None
        L.oracle_mlp_grad.argtypes = [_f32p, _u16p, _f32p, _i64, C.c_int, _f64p]
        L.oracle_mlp_grad.restype = C.c_double
        L.oracle_model_layered.argtypes = [_f32p, _i64, _i64, _i64, C.c_uint64, C.c_int,
                                           C.c_float, C.c_float, C.c_float, C.c_float,
                                           C.POINTER(C.c_float)]
        L.oracle_model_layered.restype = C.c_int
        L.oracle_mt64_nth.argtypes = [C.c_uint64, _i64]
        L.oracle_mt64_nth.restype = C.c_uint64
        L.oracle_rms_diff_f32.argtypes = [_f32p, _f32p, _i64]
        L.oracle_rms_diff_f32.restype = C.c_double
        L.oracle_max_abs_diff_f32.argtypes = [_f32p, _f32p, _i64]
        L.oracle_max_abs_diff_f32.restype = C.c_double
        _lib = L
    return _lib


def _dt(a):
    return np.float32 if a.dtype == np.float32 else np.float64


def _sfx(a):
    return "f32" if a.dtype == np.float32 else "f64"


def fd_coefficients() -> np.ndarray:
    out = np.zeros(5, np.float64)
    lib().oracle_fd_coefficients(out)
    return out


def wave_step(cur, prev, vel2, dx, dy, dz, dt, out=None):
    """One reference-order leapfrog step on (nz, ny, nx) arrays; halo of out untouched."""
    nz, ny, nx = cur.shape
    if out is None:
        out = np.zeros_like(cur)
    T = _dt(cur)
    getattr(lib(), f"oracle_wave_step_{_sfx(cur)}")(
        cur, prev, vel2, out, nx, ny, nz, T(dx), T(dy), T(dz), T(dt))
    return out


def heat_step(u, dx, dy, dz, dt_eff, alpha, out=None):
    nz, ny, nx = u.shape
    if out is None:
        out = np.zeros_like(u)
    T = _dt(u)
    getattr(lib(), f"oracle_heat_step_{_sfx(u)}")(
        u, out, nx, ny, nz, T(dx), T(dy), T(dz), T(dt_eff), T(alpha))
    return out


def wave_run(cur, prev, vel2, dx, dy, dz, dt, n_steps, src=-1, wavelet=None, trace=False):
    """n_steps of the three-level scheme in place; returns (cur, prev, trace or None)."""
    nz, ny, nx = cur.shape
    T = _dt(cur)
    scratch = np.zeros_like(cur)
    wl = None
    if wavelet is not None:
        wl = np.ascontiguousarray(wavelet, dtype=np.float64)
    tr = np.zeros(n_steps, dtype=cur.dtype) if trace else None
    getattr(lib(), f"oracle_wave_run_{_sfx(cur)}")(
        cur, prev, scratch, vel2, nx, ny, nz, T(dx), T(dy), T(dz), T(dt), n_steps, src,
        wl.ctypes.data if wl is not None else None,
        tr.ctypes.data if tr is not None else None)
    return cur, prev, tr


def wave_step_f16(P, Q, K, dx, dy, dz, m_out=1.0, m_q=1.0, src=-1, w=0.0, a=1.0, out=None):
    """One FP16-storage step (uint16 fields holding fp16 / bf16 bit patterns)."""
    nz, ny, nx = P.shape
    if out is None:
        out = Q.copy()
    lib().oracle_wave_step_f16(P, Q, K, out, nx, ny, nz, dx, dy, dz, m_out, m_q, src, w, a)
    return out


def mlp_features(p, vel2, cell, dt_over_dx):
    """(row of 32 BF16 bit patterns, scale s) of the star at flat index cell."""
    nz, ny, nx = p.shape
    row = np.zeros(32, np.uint16)
    s = lib().oracle_mlp_features(np.ascontiguousarray(p, np.float32),
                                  np.ascontiguousarray(vel2, np.float32), nx, ny, int(cell),
                                  dt_over_dx, row)
    return row, s


def mlp_forward(params, X, round_bf16=True):
    X = np.ascontiguousarray(X, np.uint16)
    y = np.zeros(X.shape[0], np.float64)
    lib().oracle_mlp_forward(np.ascontiguousarray(params, np.float32), X, X.shape[0],
                             int(round_bf16), y)
    return y


def mlp_grad(params, X, t, round_bf16=True):
    """(loss, gradient) of mean (MLP(X) - t)^2 in double."""
    X = np.ascontiguousarray(X, np.uint16)
    g = np.zeros(lib().oracle_mlp_nparam(), np.float64)
    loss = lib().oracle_mlp_grad(np.ascontiguousarray(params, np.float32), X,
                                 np.ascontiguousarray(t, np.float32), X.shape[0],
                                 int(round_bf16), g)
    return loss, g


def to_f16(a, scale=1.0) -> np.ndarray:
    """fp16 bit patterns of float32(a) * scale (round to nearest even)."""
    return (np.asarray(a, np.float32) * np.float32(scale)).astype(np.float16).view(np.uint16)


def to_bf16(a) -> np.ndarray:
    """bf16 bit patterns of float32 values (round to nearest even)."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def ricker(f, t0, dt, n_steps) -> np.ndarray:
    out = np.zeros(n_steps, np.float64)
    lib().oracle_ricker(f, t0, dt, n_steps, out)
    return out


def model_layered(nx, ny, nz, seed, n_layers=8, v_top=1500.0, v_bottom=4500.0,
                  perturbation=0.05, corr_cells=20.0):
    """Seeded layered v^2 model, (nz, ny, nx) float32, and v_max: the oracle's
    restatement of the benchmark's velocity model (model_oracle.c)."""
    out = np.empty((nz, ny, nx), np.float32)
    vmax = C.c_float()
    rc = lib().oracle_model_layered(out, nx, ny, nz, seed, n_layers, v_top, v_bottom,
                                    perturbation, corr_cells, C.byref(vmax))
    if rc != 0:
        raise ValueError("oracle_model_layered: invalid arguments")
    return out, float(vmax.value)


def mt64_nth(seed: int, n: int) -> int:
    """The n-th output (1-based) of the MT19937-64 engine seeded with `seed`."""
    return int(lib().oracle_mt64_nth(seed, n))


def rms_diff(a, b) -> float:
    return lib().oracle_rms_diff_f32(np.ascontiguousarray(a, np.float32),
                                     np.ascontiguousarray(b, np.float32), a.size)


def max_abs_diff(a, b) -> float:
    return lib().oracle_max_abs_diff_f32(np.ascontiguousarray(a, np.float32),
                                         np.ascontiguousarray(b, np.float32), a.size)


def rel_l2(a, b) -> float:
    """||a - b||_2 / ||b||_2 in double."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / nb) if nb > 0 else float(np.linalg.norm(a))


# ── the reference's own CPU path (oracle/_ref) ─────────────────────────────────

def ref_available(variant: str = "f32_strict") -> bool:
    return (HERE / "_ref" / f"libstencil_ref_{variant}.so").exists()


def ref(variant: str = "f32_strict") -> C.CDLL:
    if variant not in _ref:
        path = HERE / "_ref" / f"libstencil_ref_{variant}.so"
        L = C.CDLL(str(path))
        T = C.c_double if variant == "f64" else C.c_float
        P = _f64p if variant == "f64" else _f32p
        L.ref_real_size.restype = C.c_int
        L.ref_upload_fd_coefficients.restype = None
        L.ref_launch_naive.argtypes = [P, P, P, P, _i64, _i64, _i64, C.c_double, C.c_double,
                                       C.c_double, C.c_double]
        L.ref_launch_naive.restype = None
        L.ref_wave_run.argtypes = [P, P, P, P, _i64, _i64, _i64, C.c_double, C.c_double,
                                   C.c_double, C.c_double, _i64, _i64, C.c_void_p]
        L.ref_wave_run.restype = None
        L.ref_solver_run.argtypes = [C.c_int, _i64, C.c_double, C.c_double, C.c_double,
                                     C.c_double, C.c_int, P]
        L.ref_solver_run.restype = C.c_int
        L.ref_make_grid_dt.argtypes = [C.c_double, C.c_double]
        L.ref_make_grid_dt.restype = C.c_double
        L.ref_init_gaussian.argtypes = [P, _i64, _i64, _i64, C.c_double, C.c_double,
                                        C.c_double, C.c_double]
        L.ref_init_gaussian.restype = None
        L.ref_upload_fd_coefficients()
        _ref[variant] = L
        del T
    return _ref[variant]


def ref_wave_step(cur, prev, vel2, dx, dy, dz, dt, variant="f32_strict", out=None):
    nz, ny, nx = cur.shape
    if out is None:
        out = np.zeros_like(cur)
    ref(variant).ref_launch_naive(cur, prev, vel2, out, nx, ny, nz, dx, dy, dz, dt)
    return out


def ref_wave_run(cur, prev, vel2, dx, dy, dz, dt, n_steps, src=-1, wavelet=None,
                 variant="f32_strict"):
    nz, ny, nx = cur.shape
    scratch = np.zeros_like(cur)
    wl = None if wavelet is None else np.ascontiguousarray(wavelet, dtype=np.float64)
    ref(variant).ref_wave_run(cur, prev, scratch, vel2, nx, ny, nz, dx, dy, dz, dt, n_steps,
                              src, wl.ctypes.data if wl is not None else None)
    return cur, prev


def ref_omp_threads(variant: str = "f32") -> int:
    """OpenMP threads the reference CPU launcher uses in this process."""
    L = ref(variant)
    L.ref_omp_threads.restype = C.c_int
    return int(L.ref_omp_threads())


def ref_init_gaussian(shape, cx, cy, cz, sigma, variant="f32_strict"):
    nz, ny, nx = shape
    dt = np.float64 if variant == "f64" else np.float32
    out = np.zeros(shape, dt)
    ref(variant).ref_init_gaussian(out, nx, ny, nz, cx, cy, cz, sigma)
    return out


def ref_solver_run(physics, n, dx, velocity, diffusivity, sigma, steps, variant="f32_strict"):
    dt = np.float64 if variant == "f64" else np.float32
    out = np.zeros((n, n, n), dt)
    rc = ref(variant).ref_solver_run(physics, n, dx, velocity, diffusivity, sigma, steps, out)
    if rc != 0:
        raise RuntimeError("reference solver run failed")
    return out
