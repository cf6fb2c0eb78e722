"""Shared pytest setup.

Markers: `gpu` = needs a CUDA device (run with `-m gpu` on a B200); everything
else runs on CPU.  The CUDA path is exercised only through the C ABI of
stencil_solver_b200/lib/libstencil_b200.so; the oracle (oracle/) is the checker.
"""
from __future__ import annotations

import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the oracle and (if nvcc is present and the library is missing) the library."""
    from oracle import build as obuild

    obuild.build_oracle()
    obuild.build_reference()
    lib = ROOT / "stencil_solver_b200" / "lib" / "libstencil_b200.so"
    if not lib.exists():
        from stencil_solver_b200 import _build

        _build.build()
    obuild.build_reference_tests()
    yield


@pytest.fixture(scope="session")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch


def gaussian_field(shape, cx=0.5, cy=0.5, cz=0.5, sigma=4.0, dtype=np.float32):
    """The reference's init_gaussian (include/stencil/grid.hpp:57-78): interior-only
    Gaussian, centre at c*(n-1), halos zero, evaluated in the field's precision."""
    nz, ny, nx = shape
    T = np.dtype(dtype).type
    out = np.zeros(shape, dtype)
    icx, icy, icz = T(cx) * T(nx - 1), T(cy) * T(ny - 1), T(cz) * T(nz - 1)
    inv2s2 = T(1) / (T(2) * T(sigma) * T(sigma))
    z = np.arange(4, nz - 4, dtype=dtype)[:, None, None]
    y = np.arange(4, ny - 4, dtype=dtype)[None, :, None]
    x = np.arange(4, nx - 4, dtype=dtype)[None, None, :]
    dxx, dyy, dzz = x - icx, y - icy, z - icz
    out[4:-4, 4:-4, 4:-4] = np.exp(-(dxx * dxx + dyy * dyy + dzz * dzz) * inv2s2)
    return out
