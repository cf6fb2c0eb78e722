"""Build recipe for the oracle (test infrastructure only).

Produces
  oracle/liboracle.so                 -- the C restatements (stencil_oracle.c,
                                         model_oracle.c), -ffp-contract=off, OpenMP.
  oracle/_ref/libstencil_ref_*.so     -- the reference's own CPU path, compiled
                                         from its sources where they lie (only
                                         when the reference checkout exists):
      f32_strict : -O3 -ffp-contract=off          (bit-exact pin of the oracle)
      f32        : -O3 -march=x86-64-v4           (the reference's Release flags
                                                   with a portable -march so the
                                                   library runs on any AVX-512
                                                   host; timed CPU baseline)
      f64        : -O3 -ffp-contract=off -DSTENCIL_FP64   (FP64 CPU oracle)
The reference sources are never copied into this repository; oracle/_ref/ is
git-ignored.
"""
from __future__ import annotations

import os
import pathlib
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent

# The reference checkout this recipe compiles from: $STENCIL_REF_ROOT, else the
# path where this build environment mounts it.  Hosts without the checkout use
# prebuilt oracle/_ref/ files if they have them, and otherwise build the oracle only.
REF_ROOT = pathlib.Path(os.environ.get("STENCIL_REF_ROOT") or "/root/reference")

# Reference translation units that make up its CPU path (kernels + solver + utils).
REF_SOURCES = [
    "src/kernels/stencil_naive.cu",
    "src/kernels/stencil_tiled.cu",
    "src/utils/grid.cpp",
    "src/utils/timer.cpp",
    "src/utils/io.cpp",
    "src/solver/solver_base.cpp",
    "src/solver/wave_prop.cpp",
    "src/solver/heat_diffusion.cpp",
]

REF_VARIANTS = {
    "f32_strict": ["-O3", "-ffp-contract=off"],
    "f32": ["-O3", "-march=x86-64-v4"],
    "f64": ["-O3", "-ffp-contract=off", "-DSTENCIL_FP64"],
}


def _newer(target: pathlib.Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(pathlib.Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("oracle build failed: " + " ".join(map(str, cmd)))


def build_oracle(force: bool = False) -> pathlib.Path:
    out = HERE / "liboracle.so"
    srcs = [HERE / "stencil_oracle.c", HERE / "model_oracle.c"]
    if force or _newer(out, srcs):
        _run(["gcc", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared", "-std=c11",
              "-Wall", "-Wextra", *map(str, srcs), "-o", str(out), "-lm"])
    return out


def reference_available() -> bool:
    return all((REF_ROOT / s).exists() for s in REF_SOURCES)


def build_reference(force: bool = False) -> dict:
    """Compile the reference CPU path; returns {variant: path}. No-op without the checkout."""
    built = {}
    if not reference_available():
        return built
    outdir = HERE / "_ref"
    outdir.mkdir(exist_ok=True)
    shim = HERE / "ref_shim.cpp"
    srcs = [REF_ROOT / s for s in REF_SOURCES]
    for name, flags in REF_VARIANTS.items():
        out = outdir / f"libstencil_ref_{name}.so"
        if force or _newer(out, [shim, *srcs]):
            cmd = ["g++", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-w",
                   "-DSTENCIL_CPU_FALLBACK", *flags, "-I", str(REF_ROOT / "include")]
            for s in srcs:
                cmd += ["-x", "c++", str(s)]
            cmd += ["-x", "c++", str(shim), "-o", str(out)]
            _run(cmd)
        built[name] = out
    return built


# The reference's own test sources, compiled unchanged against the B200
# library's drop-in headers (include/stencil/) and libstencil_b200.so, on the
# GoogleTest-compatible shim in tests/cpp/gtest_shim.  CPU ones only need the
# library to load; GPU ones exercise the kernels and solvers.
REF_TESTS_CPU = ["tests/unit/test_fd_coeffs.cpp", "tests/unit/test_grid.cpp",
                 "tests/unit/test_timer.cpp", "tests/unit/test_io.cpp",
                 "tests/unit/test_solver_cpu.cpp"]
REF_TESTS_GPU = ["tests/unit/test_kernels.cpp", "tests/unit/test_solver.cpp",
                 "tests/integration/test_kernel_correctness.cpp",
                 "tests/integration/test_wave_3d.cpp", "tests/integration/test_heat_3d.cpp"]


def reference_test_binary(src: str) -> pathlib.Path:
    return HERE / "_ref" / ("reftest_" + pathlib.Path(src).stem)


def build_reference_tests(force: bool = False) -> list:
    """Builds oracle/_ref/reftest_* (needs the reference checkout and the library)."""
    repo = HERE.parent
    lib = repo / "stencil_solver_b200" / "lib" / "libstencil_b200.so"
    if not lib.exists() or not all((REF_ROOT / s).exists() for s in REF_TESTS_CPU + REF_TESTS_GPU):
        return []
    (HERE / "_ref").mkdir(exist_ok=True)
    shim = repo / "tests" / "cpp" / "gtest_shim"
    headers = list((repo / "include" / "stencil").glob("*")) + [shim / "gtest" / "gtest.h"]
    out = []
    for src in REF_TESTS_CPU + REF_TESTS_GPU:
        exe = reference_test_binary(src)
        deps = [REF_ROOT / src, shim / "gtest_main.cpp", lib, *headers]
        if force or _newer(exe, deps):
            _run(["nvcc", "-std=c++17", "-O2", "-w", "-I", str(repo / "include"), "-I", str(shim),
                  str(REF_ROOT / src), str(shim / "gtest_main.cpp"), "-o", str(exe),
                  "-L", str(lib.parent), "-lstencil_b200",
                  "-Xlinker", "-rpath,$ORIGIN/../../stencil_solver_b200/lib"])
        out.append(exe)
    return out


def build(force: bool = False) -> None:
    build_oracle(force)
    build_reference(force)
    build_reference_tests(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print("oracle built:", HERE / "liboracle.so")
    for p in sorted((HERE / "_ref").glob("*.so")) if (HERE / "_ref").exists() else []:
        print("reference CPU path built:", p)
