"""The reference's own unit and integration tests, compiled unchanged against the
B200 drop-in headers (include/stencil/) and libstencil_b200.so.

The binaries are built by oracle/build.py (build_reference_tests) from the
reference's test sources into oracle/_ref/ on the GoogleTest-compatible shim in
tests/cpp/gtest_shim; they travel with the tree, so the GPU half runs on a box
without the reference checkout.
"""
from __future__ import annotations

import pathlib
import subprocess

import pytest

from oracle import build as obuild

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _run(exe: pathlib.Path, tmp_path) -> subprocess.CompletedProcess:
    return subprocess.run([str(exe)], cwd=tmp_path, capture_output=True, text=True, timeout=600)


def _binary(src):
    exe = obuild.reference_test_binary(src)
    if not exe.exists():
        obuild.build_reference_tests()
    if not exe.exists():
        pytest.skip("reference test binaries not built (no reference checkout)")
    return exe


def test_shim_reports_planted_failures(tmp_path):
    shim = ROOT / "tests" / "cpp" / "gtest_shim"
    exe = tmp_path / "shim_selftest"
    subprocess.run(["g++", "-std=c++17", "-I", str(shim), str(ROOT / "tests/cpp/shim_selftest.cpp"),
                    str(shim / "gtest_main.cpp"), "-o", str(exe)], check=True)
    r = _run(exe, tmp_path)
    assert r.returncode == 1
    assert "4 tests ran, 3 failed" in r.stdout
    assert "[       OK ] ShimSelfTest.Passes" in r.stdout
    assert "planted" in r.stderr


@pytest.mark.parametrize("src", obuild.REF_TESTS_CPU)
def test_reference_cpu_suite(src, tmp_path):
    r = _run(_binary(src), tmp_path)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert " 0 failed" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("src", obuild.REF_TESTS_GPU)
def test_reference_gpu_suite(src, tmp_path):
    r = _run(_binary(src), tmp_path)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert " 0 failed" in r.stdout
