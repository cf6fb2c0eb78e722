"""Learned 2x-coarse stepping: training pairs from the plain fine solver, training
of the correction network on the GPU, and the coarse run it corrects.

No reference counterpart (the reference solves on one grid only).  Geometry:
a coarse grid of nc points per axis at spacing h and time step dt pairs with a
fine grid of 2 nc - 8 points at h / 2 and dt / 2, aligned so that coarse cell i
sits on fine cell 2 i - 4.  Both grids then have their interior start and their
far wall at the same physical positions (the near wall differs by half a coarse
cell).

Source: both grids discretise the same continuum term S(x, t) = A v^2 w(t) g(x),
w a Ricker wavelet and g a Gaussian of width sigma (2 coarse cells by default)
around the source point: each step adds dt^2 S(x_j, t_n) on a box of cells
(the coarse grid's w samples are the [1, 2, 1] / 4 average of the fine ones,
see Problem.wavelet).  Two fine leapfrog steps of h = dt / 2 compose to

    p(t + 2h) - 2 p(t) + p(t - 2h) = (2h)^2 [L p + S-bar] + h^4 L^2 p + h^4 L S(t),

L = v^2 lap and S-bar the [1, 2, 1] / 4 average: the coarse step has the first
term; the network learns the h^4 L^2 p part of the rest (a function of the
state); the coarse source adds the state-independent h^4 L S(t) term, computed
once as the pattern v^2 lap(v^2 g) on the coarse grid (Problem.source).  A
point source (the reference's rule, one cell) puts energy above the coarse
grid's Nyquist wavenumber, which no coarse state can represent; the Gaussian
keeps the field band-limited, so the coarse-grid error is the scheme's
dispersion error, a function of the local state.

Velocity: the coarse grid samples the fine model.  A sharply layered model is a
different medium on the two grids (an interface moves by up to half a coarse
cell), so `smooth_cells` > 0 first smooths the fine model with a Gaussian of
that width (in coarse cells; sb200_smooth3 on the device): the medium both
grids resolve.

Training pairs (coarse state at t, fine state at t + dt restricted): with C_m
the restriction of the fine field after 2m fine steps, the plain coarse step
from (C_{m-1}, C_{m-2}) gives P_m; the network learns (C_m - P_m) / s from the
features of C_{m-1} (see stencil_b200.h, sb200_mlp_*).

The host loop here only orders C-ABI calls on device buffers (torch allocates
them); every operation on field data is a kernel of the library.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import NamedTuple

import numpy as np

from . import (Grid, Mlp, _check, add_box, lib, mlp_samples, restrict2, smooth3, wave_prepass,
               wave_step)

OFFSET = -4  # coarse cell i <-> fine cell 2 i + OFFSET
# Correction floor of a trained network (Mlp.min_scale).  A Problem's source is
# normalised so that its fields are O(1); points whose star stays below 2^-24 of
# that get no correction, so the values the stencil leaves ahead of the wavefront
# decay and underflow as in the plain solve (a correction proportional to them
# would keep the whole numerical light cone, 4 cells per step, nonzero).  The
# omitted corrections are ~1e-9 of the field; a higher floor also leaves fewer
# chunks on the fused step's network path (516^3, 200 steps: 2^-64 95 ms,
# 2^-40 92 ms, 2^-24 90 ms, the same errors).
CORRECTION_FLOOR = 2.0 ** -24


def _torch():
    import torch

    return torch


def fine_extent(nc: int) -> int:
    return 2 * nc - 8


# 8th-order central second-derivative weights (the library's FD coefficients)
_FD8 = (-205.0 / 72, 8.0 / 5, -1.0 / 5, 8.0 / 315, -1.0 / 560)


class Source(NamedTuple):
    """A grid's source term: each step adds dt^2 amp w pattern on the box
    (origin (x, y, z), dims); on the coarse grid also h^4 amp w(t) comp_pattern
    on the box (comp_origin, comp_dims), h the fine step (the composition term)."""
    origin: tuple
    dims: tuple
    pattern: object
    amp: float
    comp_origin: tuple = None
    comp_dims: tuple = None
    comp_pattern: object = None

    def box(self) -> tuple:
        """(x0, x1, y0, y1, z0, z1): the cells the source writes (both boxes)."""
        lo = list(self.origin)
        hi = [o + d for o, d in zip(self.origin, self.dims)]
        if self.comp_pattern is not None:
            lo = [min(a, b) for a, b in zip(lo, self.comp_origin)]
            hi = [max(a, o + d) for a, o, d in zip(hi, self.comp_origin, self.comp_dims)]
        return (lo[0], hi[0], lo[1], hi[1], lo[2], hi[2])


@dataclass
class Problem:
    """One velocity model on the coarse / fine pair of grids."""
    nc: int
    h: float            # coarse spacing [m]
    dt: float           # coarse time step [s]
    seed: int
    freq: float = 25.0
    src_c: tuple = None  # source point in coarse cells (x, y, z); default: the centre
    sigma_cells: float = 2.0  # source width in coarse cells
    model: str = "layered"    # "layered" or "constant"
    smooth_cells: float = 0.0  # Gaussian smoothing of the fine model, in coarse cells
    layers: int = 8
    v_top: float = 1500.0
    v_bottom: float = 4500.0
    perturbation: float = 0.05
    corr_cells: float = 20.0
    vel2_window: object = None  # device fine model to use instead of generating one
    compose_source: bool = True  # the coarse source's h^4 L S term (see the module doc)
    compose_state: bool = False  # the coarse step's h^4 L^2 p term (coarse_step)

    def __post_init__(self):
        if self.src_c is None:
            c = self.nc // 2
            self.src_c = (c, c, c)
        self._vf = self._vc = None
        self._wc = None  # cached wavelet_centre samples

    @property
    def coarse(self) -> Grid:
        return Grid(self.nc, self.nc, self.nc, self.h, self.h, self.h, self.dt)

    @property
    def fine(self) -> Grid:
        nf = fine_extent(self.nc)
        return Grid(nf, nf, nf, self.h / 2, self.h / 2, self.h / 2, self.dt / 2)

    def wavelet(self, fine: bool, n: int) -> np.ndarray:
        """Source samples of the first n steps.  Fine: w(k dt_f).  Coarse:
        (w(t - dt_f) + 2 w(t) + w(t + dt_f)) / 4 at t = m dt_c -- two fine
        leapfrog steps add up to one coarse step whose source term is exactly
        that [1, 2, 1] / 4 average of the fine samples, so the coarse grid
        injects what the fine grid does, to the scheme's order."""
        dtf = self.fine.dt
        if fine:
            w = np.empty(n, np.float32)
            _check(lib().sb200_ricker(self.freq, 1.0 / self.freq, dtf, n, w.ctypes.data))
            return w
        s = np.empty(2 * n + 2, np.float32)  # s[k] = w((k - 1) dt_f)
        _check(lib().sb200_ricker(self.freq, 1.0 / self.freq + dtf, dtf, 2 * n + 2,
                                  s.ctypes.data))
        s = s.astype(np.float64)
        return ((s[0:2 * n:2] + 2 * s[1:2 * n + 1:2] + s[2:2 * n + 2:2]) / 4).astype(np.float32)

    def vel2_fine_host(self) -> np.ndarray:
        """The unsmoothed fine model: seeded layered (host generator of the
        library) or constant (a seeded speed in [v_top, v_bottom])."""
        g = self.fine
        if self.model == "constant":
            v = np.random.default_rng(self.seed).uniform(self.v_top, self.v_bottom)
            return np.full(g.shape, v * v, np.float32)
        v2 = np.empty(g.shape, np.float32)
        vmax = C.c_float()
        _check(lib().sb200_model_layered(v2.ctypes.data, g.nx, g.ny, g.nz, self.seed, self.layers,
                                         self.v_top, self.v_bottom, self.perturbation,
                                         self.corr_cells, C.byref(vmax)))
        return v2

    def device_models(self):
        """(vel2 fine, vel2 coarse) on the device, built once: the fine model,
        smoothed by smooth_cells coarse cells (sb200_smooth3), and its
        restriction to the coarse grid."""
        if self._vf is None:
            torch = _torch()
            if self.vel2_window is not None:
                vf = self.vel2_window
            else:
                vf = torch.from_numpy(self.vel2_fine_host()).cuda()
            if self.smooth_cells > 0 and self.vel2_window is None:
                tmp = torch.empty_like(vf)
                smooth3(vf, tmp, self.fine, 2.0 * self.smooth_cells)
                del tmp
            vc = torch.empty(self.coarse.shape, device="cuda")
            restrict2(vf, self.fine, vc, self.coarse, OFFSET)
            self._vf, self._vc = vf, vc
        return self._vf, self._vc

    def release(self) -> None:
        """Drops the cached device models."""
        self._vf = self._vc = None
        self._wc = None  # cached wavelet_centre samples

    def wavelet_centre(self, n: int) -> np.ndarray:
        """w(t_m) at the first n coarse times t_m = m dt (the centre sample of the
        coarse [1, 2, 1] / 4 average): the fine samples of even index."""
        return self.wavelet(True, 2 * n)[0::2]

    def source(self, fine: bool) -> Source:
        """The grid's Source: pattern_j = vel2_j g(x_j) on the box of cells within
        3.5 sigma of the source point, amplitude A; on the coarse grid also the
        composition pattern vel2 lap(vel2 g) (8th-order Laplacian of the coarse
        grid) on that box widened by the stencil radius."""
        torch = _torch()
        vf, vc = self.device_models()
        sig = self.sigma_cells  # in coarse cells
        rad_c = int(math.ceil(3.5 * sig))
        if fine:
            v = vf
            centre = [2 * c + OFFSET for c in self.src_c]
            rad, unit = 2 * rad_c + 1, 0.5  # a fine cell is half a coarse cell
        else:
            v = vc
            centre = list(self.src_c)
            rad, unit = rad_c, 1.0
        origin = [c - rad for c in centre]
        n = 2 * rad + 1
        off = (np.arange(n) - rad) * unit
        r2 = off[None, None, :] ** 2 + off[None, :, None] ** 2 + off[:, None, None] ** 2
        gx = np.exp(-r2 / (2 * sig * sig))
        zs, ys, xs = [slice(o, o + n) for o in origin[::-1]]
        box = v[zs, ys, xs].cpu().numpy().astype(np.float64)
        pat = (box * gx).astype(np.float32)
        amp = 1.0 / (self.dt * self.dt * 3000.0 * 3000.0)  # O(1) fields
        pat_d = torch.from_numpy(np.ascontiguousarray(pat)).cuda()
        if fine or not self.compose_source:
            return Source(tuple(origin), (n, n, n), pat_d, amp)
        # v^2 lap(v^2 g) on the box widened by 4; v^2 g on a box widened by 8
        # (cells outside the grid take the nearest edge value of v^2)
        R = 4
        ext = rad + 2 * R
        idx = [np.clip(np.arange(c - ext, c + ext + 1), 0, d - 1)
               for c, d in zip(centre[::-1], v.shape)]
        iz, iy, ix = (torch.as_tensor(i, device=v.device) for i in idx)
        vbox = v.index_select(0, iz).index_select(1, iy).index_select(2, ix)
        vbox = vbox.cpu().numpy().astype(np.float64)
        offe = np.arange(2 * ext + 1) - ext
        r2e = offe[None, None, :] ** 2 + offe[None, :, None] ** 2 + offe[:, None, None] ** 2
        u = vbox * np.exp(-r2e / (2 * sig * sig))
        lap = 3 * _FD8[0] * u
        for r in range(1, R + 1):
            for ax in range(3):
                lap = lap + _FD8[r] * (np.roll(u, r, ax) + np.roll(u, -r, ax))
        inner = slice(R, 2 * ext + 1 - R)
        comp = (vbox * lap / (self.h * self.h))[inner, inner, inner].astype(np.float32)
        nw = comp.shape[0]
        return Source(tuple(origin), (n, n, n), pat_d, amp,
                      tuple(c - rad - R for c in centre), (nw, nw, nw),
                      torch.from_numpy(np.ascontiguousarray(comp)).cuda())


def _inject(pb: Problem, fine: bool, fld, src: Source, w, k) -> None:
    g = pb.fine if fine else pb.coarse
    add_box(fld, g, src.origin, src.dims, src.pattern, float(g.dt * g.dt * src.amp * w[k]))
    if src.comp_pattern is not None:
        h = pb.fine.dt
        wc = pb._wc if pb._wc is not None and pb._wc.size > k else pb.wavelet_centre(2 * k + 64)
        pb._wc = wc
        add_box(fld, g, src.comp_origin, src.comp_dims, src.comp_pattern,
                float(h ** 4 * src.amp * wc[k]))


def fine_solve(pb: Problem, vf, steps: int, on_even=None):
    """Plain fine solve from rest for `steps` fine steps.  on_even(m, field) is
    called after every even number 2m of steps (m >= 0) with the device field."""
    torch = _torch()
    g = pb.fine
    p = torch.zeros(g.shape, device="cuda")
    q = torch.zeros(g.shape, device="cuda")
    w = pb.wavelet(True, steps)
    src = pb.source(True)
    if on_even:
        on_even(0, p)
    for n in range(steps):
        wave_step(p, q, vf, q, g)
        _inject(pb, True, q, src, w, n)
        p, q = q, p
        if on_even and (n + 1) % 2 == 0:
            on_even((n + 1) // 2, p)
    return p


def coarse_step(pb: Problem, vc, p, q, src, w, m, mlp: Mlp | None = None,
                fused: bool = True, flags=None, r=None):
    """One coarse step from level m (p) over level m-1 (q, overwritten with m+1):
    the acoustic step, the learned correction (mlp given; one fused launch unless
    fused is False), then the source.  flags = (flags of p, flags for q): the
    fused step's activity flags (chunks far from any value at the correction
    floor skip the network; the source box counts as active); with
    pb.compose_state a third buffer, the scratch for the flags of r.

    With pb.compose_state the step first runs the pre-pass
    (sb200_wave_prepass_f32, beta = 1/16) into the scratch field r (zero halo):
    r = p + (dt^2 / 16) L p and q += (dt^2 / 8) L p, and then steps (r, q), which
    adds the composition term h^4 L^2 p of two fine steps (h = dt / 2).  The
    network then sees the stars of r.  Returns the field that was stepped."""
    g = pb.coarse
    cur = p
    box = None if flags is None else src.box()
    if pb.compose_state:
        if r is None:
            raise ValueError("coarse_step: compose_state needs the scratch field r")
        wave_prepass(p, q, vc, r, g, 1.0 / 16.0)
        cur = r
        if flags is not None and mlp is not None and fused:
            # flags = (flags of p, flags for q, scratch for the flags of r)
            mlp.flags_compose(g, flags[0], flags[2])
            flags = (flags[2], flags[1])
            box = tuple(b + (4 if k % 2 else -4) for k, b in enumerate(box))
    if mlp is None:
        wave_step(cur, q, vc, q, g)
    elif fused:
        mlp.learned_step(cur, q, vc, g, flags=flags, box=box)
    else:
        wave_step(cur, q, vc, q, g)
        mlp.correct(cur, vc, q, g)
    _inject(pb, False, q, src, w, m)
    return cur


def new_flags(mlp: Mlp, g: Grid, compose: bool = False):
    """Activity-flag buffers for the fused step on g, every bit set (every chunk
    and face active): the pair that alternates between p and q, and with
    `compose` a third, the scratch for the flags of the pre-pass field r."""
    torch = _torch()
    n = mlp.flags_bytes(g)
    return [torch.full((n,), 255, dtype=torch.uint8, device="cuda")
            for _ in range(3 if compose else 2)]


def _flag_args(fl):
    return None if fl is None else tuple(fl)


def _rotate(fl):
    if fl is not None:
        fl[0], fl[1] = fl[1], fl[0]


def coarse_solve(pb: Problem, vc, steps: int, mlp: Mlp | None = None, use_flags: bool = True):
    """Plain (mlp None) or corrected coarse solve from rest for `steps` coarse steps
    (corrected: with activity flags unless use_flags is False; the same bits)."""
    torch = _torch()
    g = pb.coarse
    p = torch.zeros(g.shape, device="cuda")
    q = torch.zeros(g.shape, device="cuda")
    r = torch.zeros(g.shape, device="cuda") if pb.compose_state else None
    w = pb.wavelet(False, steps)
    src = pb.source(False)
    fl = new_flags(mlp, g, pb.compose_state) if mlp is not None and use_flags else None
    for m in range(steps):
        coarse_step(pb, vc, p, q, src, w, m, mlp, flags=_flag_args(fl), r=r)
        p, q = q, p
        _rotate(fl)
    return p


@dataclass
class Dataset:
    X: object  # (n, 32) int16 BF16 bit patterns, device
    t: object  # (n,) float32, device
    per_model: list = field(default_factory=list)

    @property
    def n(self) -> int:
        return int(self.t.numel())


def make_pairs(problems, fine_steps: int, samples_per_pair: int = 4096, every: int = 4,
               first: int = 8, wall: int = 12, amp_floor: float = 0.05, src_clear: float = 0.0,
               seed: int = 0) -> Dataset:
    """Training rows from the plain fine solver on each problem: every `every`
    coarse steps from `first` on, samples_per_pair random coarse cells at least
    `wall` cells from the walls and src_clear source widths from the source point,
    whose local field exceeds amp_floor x the field's largest magnitude (where
    the field is small its round-off dominates the normalised residual, which is
    then not a function of the local state).  With the coarse source's
    composition term (Problem.compose_source) the residual inside the source is
    a function of the state too, and rows there (src_clear 0) halve the
    corrected solve's early error."""
    torch = _torch()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    Xs, ts, counts = [], [], []
    for pb in problems:
        vf, vc = pb.device_models()
        gc = pb.coarse
        w_c = pb.wavelet(False, fine_steps // 2 + 2)
        src_c = pb.source(False)
        ring = {}
        plain = torch.empty(gc.shape, device="cuda")
        rbuf = torch.zeros(gc.shape, device="cuda") if pb.compose_state else None
        nz, ny, nx = gc.shape
        box = torch.zeros(gc.shape, dtype=torch.bool, device="cuda")
        box[wall:nz - wall, wall:ny - wall, wall:nx - wall] = True
        zz, yy, xx = torch.meshgrid(*(torch.arange(k, device="cuda") for k in (nz, ny, nx)),
                                    indexing="ij")
        sx, sy, sz = pb.src_c
        d2 = (xx - sx) ** 2 + (yy - sy) ** 2 + (zz - sz) ** 2
        box &= d2 > (src_clear * pb.sigma_cells) ** 2
        del zz, yy, xx, d2
        before = sum(x.shape[0] for x in Xs)

        def on_even(m, f):
            c = torch.empty(gc.shape, device="cuda")
            restrict2(f, pb.fine, c, gc, OFFSET)
            ring[m] = c
            ring.pop(m - 3, None)
            if m >= max(first, 2) and (m - first) % every == 0:
                cm2, cm1, cm = ring[m - 2], ring[m - 1], ring[m]
                plain.copy_(cm2)  # in-place leapfrog writes over the older level
                stepped = coarse_step(pb, vc, cm1, plain, src_c, w_c, m - 1, r=rbuf)
                sample_rows(stepped, cm, m)

        def sample_rows(state, target, m):
            """Rows at random cells of `state` (level m - 1); `plain` holds its plain step."""
            mag = state.abs()
            ok = box & (mag > amp_floor * float(mag.max()))
            cand = torch.nonzero(ok.view(-1)).view(-1)
            if cand.numel() == 0:
                return
            k = min(samples_per_pair, cand.numel())
            pick = cand[torch.randint(0, cand.numel(), (k,), generator=gen, device="cuda")]
            X = torch.empty((pick.numel(), 32), dtype=torch.int16, device="cuda")
            t = torch.empty(pick.numel(), dtype=torch.float32, device="cuda")
            mlp_samples(state, vc, target, plain, gc, pick.to(torch.int64), X, t)
            Xs.append(X)
            ts.append(t)

        fine_solve(pb, vf, fine_steps, on_even)
        counts.append(sum(x.shape[0] for x in Xs) - before)
        del vf, vc
        pb.release()
    return Dataset(torch.cat(Xs), torch.cat(ts), counts)


def train(ds: Dataset, mlp: Mlp, epochs: int = 4, batch: int = 8192, lr: float = 2e-3,
          lr_final: float = 1e-4, seed: int = 0, log=None) -> list:
    """Adam over shuffled mini-batches with a cosine learning-rate decay.  The
    targets are divided by their RMS, which becomes the network's output scale;
    the network's correction floor becomes CORRECTION_FLOOR.  Returns the mean
    batch loss (in units of that RMS squared) of every epoch."""
    torch = _torch()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    n = ds.n
    rms = float(ds.t.double().pow(2).mean().sqrt())
    mlp.output_scale = rms if rms > 0 else 1.0
    mlp.min_scale = CORRECTION_FLOOR
    tn = ds.t / mlp.output_scale
    steps_per_epoch = max(1, n // batch)
    total = epochs * steps_per_epoch
    loss = torch.zeros(1, device="cuda")
    acc = torch.zeros(1, device="cuda")
    history = []
    k = 0
    for ep in range(epochs):
        perm = torch.randperm(n, generator=gen, device="cuda")
        acc.zero_()
        for b in range(steps_per_epoch):
            idx = perm[b * batch:(b + 1) * batch]
            X = ds.X.index_select(0, idx)
            t = tn.index_select(0, idx)
            cur = lr_final + 0.5 * (lr - lr_final) * (1 + math.cos(math.pi * k / max(1, total - 1)))
            mlp.train_step(X, t, cur, loss)
            acc += loss
            k += 1
        history.append(float(acc.item()) / steps_per_epoch)
        if log:
            log(f"epoch {ep}: loss {history[-1]:.4e}")
    return history


def rel_l2(a, b) -> float:
    """||a - b|| / ||b|| over the interior, in double."""
    torch = _torch()
    a = a[4:-4, 4:-4, 4:-4].double()
    b = b[4:-4, 4:-4, 4:-4].double()
    nb = torch.linalg.vector_norm(b)
    return float(torch.linalg.vector_norm(a - b) / nb) if float(nb) > 0 else float("nan")


def evaluate(pb: Problem, coarse_steps: int, mlp: Mlp | None):
    """Errors of the plain and the corrected coarse solves against the restricted
    plain fine solve (the judge) after coarse_steps steps: {"plain": e0, "learned": e1}."""
    torch = _torch()
    vf, vc = pb.device_models()
    judge_f = fine_solve(pb, vf, 2 * coarse_steps)
    judge = torch.empty(pb.coarse.shape, device="cuda")
    restrict2(judge_f, pb.fine, judge, pb.coarse, OFFSET)
    del judge_f, vf
    out = {"plain": rel_l2(coarse_solve(pb, vc, coarse_steps), judge)}
    if mlp is not None:
        out["learned"] = rel_l2(coarse_solve(pb, vc, coarse_steps, mlp), judge)
    return out


def proxy_of(pb: Problem, nc_proxy: int = 64) -> Problem:
    """A small pair of grids cut from pb's (smoothed) fine model around its
    source, with the source at its centre: the judge's test problem."""
    torch = _torch()
    vf, _ = pb.device_models()
    nfp = fine_extent(nc_proxy)
    cp = nc_proxy // 2
    starts = []
    for s_ax, n_f in zip(pb.src_c[::-1], pb.fine.shape):  # z, y, x
        w0 = 2 * (s_ax - cp)  # even: coarse cells of the window line up with pb's
        w0 = max(0, min(w0 - w0 % 2, (n_f - nfp) - (n_f - nfp) % 2))
        starts.append(w0)
    z0, y0, x0 = starts
    win = vf[z0:z0 + nfp, y0:y0 + nfp, x0:x0 + nfp].contiguous()
    src = (pb.src_c[0] - x0 // 2, pb.src_c[1] - y0 // 2, pb.src_c[2] - z0 // 2)
    return Problem(nc_proxy, pb.h, pb.dt, pb.seed, freq=pb.freq, src_c=src,
                   sigma_cells=pb.sigma_cells, vel2_window=win, compose_source=pb.compose_source,
                   compose_state=pb.compose_state)


@dataclass
class SolveReport:
    steps: int                # coarse steps asked for
    fallback_at: object       # coarse step at which the judge tripped, or None
    checks: list              # (coarse step, proxy rel L2 of the corrected solve, of the plain one)
    ms: float                 # device time of the whole solve
    field: object             # result on the coarse grid (restricted fine solve after a fallback)
    network_off_at: object = None  # coarse step after which the network was switched off, or None


def proxy_extent(pb: Problem, coarse_steps: int, vmax: float) -> int:
    """Coarse extent of a proxy window that the waves from the source do not cross
    within coarse_steps steps at speed vmax (the source's reach plus 8 cells of
    margin on each side), a multiple of 8, at most the problem's own extent.  Its
    walls must stay out of reach: the coarse and fine grids' near walls sit half a
    coarse cell apart, so reflections there differ between them."""
    reach = coarse_steps * vmax * pb.dt / pb.h + 3.5 * pb.sigma_cells + 8.0
    n = int(math.ceil((2.0 * reach + 8.0) / 8.0)) * 8
    return max(32, min(n, pb.nc))


def learned_solve(pb: Problem, coarse_steps: int, mlp: Mlp, bound: float = 1e-3,
                  check_every: int = 20, nc_proxy: int | None = None,
                  rival: bool = True) -> SolveReport:
    """Corrected coarse solve with the plain fine solver as judge and fallback.

    A proxy pair (proxy_of) is advanced alongside the main coarse solve: its
    plain fine solve (2 steps per coarse step), its corrected coarse solve and,
    with `rival`, its coarse solve without the network.  Every check_every
    coarse steps the proxy's coarse fields are compared with its restricted fine
    field.  When the corrected proxy is further from the fine one than the
    uncorrected one, the network is switched off for the rest of the solve (main
    and proxy); when the proxy of the method in use exceeds `bound`, the coarse
    solve is abandoned and the plain fine solve computes the answer.  Device time
    (CUDA events) covers everything, fallback included.  nc_proxy None: the
    proxy_extent of the solve."""
    torch = _torch()
    vf, vc = pb.device_models()
    if nc_proxy is None:
        nc_proxy = proxy_extent(pb, coarse_steps, float(vc.max().sqrt()))
    px = proxy_of(pb, nc_proxy)
    pvf, pvc = px.device_models()
    e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
    torch.cuda.synchronize()
    e0.record()
    g, gp, gpf = pb.coarse, px.coarse, px.fine
    p = torch.zeros(g.shape, device="cuda")
    q = torch.zeros(g.shape, device="cuda")
    pp = torch.zeros(gp.shape, device="cuda")
    pq = torch.zeros(gp.shape, device="cuda")
    rp = torch.zeros(gp.shape, device="cuda") if rival else None  # proxy without the network
    rq = torch.zeros(gp.shape, device="cuda") if rival else None
    fp = torch.zeros(gpf.shape, device="cuda")
    fq = torch.zeros(gpf.shape, device="cuda")
    judge = torch.empty(gp.shape, device="cuda")
    r = torch.zeros(g.shape, device="cuda") if pb.compose_state else None
    pr = torch.zeros(gp.shape, device="cuda") if pb.compose_state else None
    w = pb.wavelet(False, coarse_steps)
    wp = px.wavelet(False, coarse_steps)
    wf = px.wavelet(True, 2 * coarse_steps)
    src, psrc, pfsrc = pb.source(False), px.source(False), px.source(True)
    fl, pfl = new_flags(mlp, g, pb.compose_state), new_flags(mlp, gp, pb.compose_state)
    net = mlp
    checks, fallback, off_at = [], None, None
    for m in range(coarse_steps):
        coarse_step(pb, vc, p, q, src, w, m, net, flags=_flag_args(fl) if net else None, r=r)
        p, q = q, p
        _rotate(fl)
        coarse_step(px, pvc, pp, pq, psrc, wp, m, net, flags=_flag_args(pfl) if net else None, r=pr)
        pp, pq = pq, pp
        _rotate(pfl)
        if rival and net is not None:
            coarse_step(px, pvc, rp, rq, psrc, wp, m, None, r=pr)
            rp, rq = rq, rp
        for k in (2 * m, 2 * m + 1):
            wave_step(fp, fq, pvf, fq, gpf)
            _inject(px, True, fq, pfsrc, wf, k)
            fp, fq = fq, fp
        if (m + 1) % check_every == 0 or m + 1 == coarse_steps:
            restrict2(fp, gpf, judge, gp, OFFSET)
            err = rel_l2(pp, judge)
            err_rival = rel_l2(rp, judge) if rival and net is not None else None
            checks.append((m + 1, err, err_rival))
            if err_rival is not None and err_rival < err:
                # the network loses on the proxy: carry on without it from the
                # uncorrected proxy state (its history is the uncorrected one)
                net, off_at = None, m + 1
                pp.copy_(rp)
                pq.copy_(rq)
                err = err_rival
            if err > bound:
                fallback = m + 1
                break
    if fallback is not None:
        del p, q
        ff = fine_solve(pb, vf, 2 * coarse_steps)
        p = torch.empty(g.shape, device="cuda")
        restrict2(ff, pb.fine, p, g, OFFSET)
        del ff
    e1.record()
    torch.cuda.synchronize()
    return SolveReport(coarse_steps, fallback, checks, e0.elapsed_time(e1), p, off_at)


def time_fine_solve(pb: Problem, fine_steps: int):
    """(device ms, restricted result) of the plain fine solve.  Two untimed steps
    first, so the pencil tuner's first-use work stays outside."""
    torch = _torch()
    vf, _ = pb.device_models()
    fine_solve(pb, vf, 2)
    e0, e1 = torch.cuda.Event(True), torch.cuda.Event(True)
    torch.cuda.synchronize()
    e0.record()
    f = fine_solve(pb, vf, fine_steps)
    e1.record()
    torch.cuda.synchronize()
    out = torch.empty(pb.coarse.shape, device="cuda")
    restrict2(f, pb.fine, out, pb.coarse, OFFSET)
    return e0.elapsed_time(e1), out
