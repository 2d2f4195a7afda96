"""Host code under AddressSanitizer and UndefinedBehaviorSanitizer. CPU only.

The geometry builders (csrc/geometry.cpp) make every table the device kernels
index: chroma axes and their bilinear axes, polyphase luma tables, radial
phase tables, lc footprint extents and rescue factors. The sweep in
host_sanitize/geometry_sweep.cpp builds them over degenerate and real sizes,
all kernel profiles, sitings, ratios and resize directions in a binary
compiled with -fsanitize=address,undefined, and checks the index ranges and
sizes the kernels rely on. (The device side of the same plan is the
poisoned-workspace GPU test.)
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "vapoursynth-lgcr_b200", "csrc")
SWEEP = os.path.join(ROOT, "tests", "host_sanitize", "geometry_sweep.cpp")
OUT_DIR = os.path.join(ROOT, "tests", "_build")


def build_sweep():
    """Compile the sweep with the first C++ compiler here whose sanitizer
    runtime links ($CXX, then g++ and clang++ on PATH)."""
    os.makedirs(OUT_DIR, exist_ok=True)
    exe = os.path.join(OUT_DIR, "geometry_sweep_asan")
    tried = []
    for cxx in dict.fromkeys(c for c in (os.environ.get("CXX"), "g++", "clang++") if c):
        if shutil.which(cxx) is None:
            continue
        cmd = [cxx, "-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer",
               "-fsanitize=address,undefined", "-fno-sanitize-recover=all", "-ffp-contract=off",
               "-I", CSRC, os.path.join(CSRC, "geometry.cpp"), SWEEP, "-o", exe]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode == 0:
            return exe
        if "error:" in r.stderr and "ld returned" not in r.stderr:
            raise AssertionError(f"sweep did not compile with {cxx}:\n" + r.stderr[-3000:])
        tried.append(f"{cxx}: " + r.stderr.strip().splitlines()[-1])
    pytest.skip("no compiler with a linkable sanitizer runtime (" + "; ".join(tried) + ")")


def test_geometry_tables_under_asan_ubsan():
    exe = build_sweep()
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:halt_on_error=1",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1")
    r = subprocess.run([exe], capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr[-4000:]
    assert " 0 failures" in r.stdout, r.stdout
    assert "runtime error" not in r.stderr, r.stderr[-4000:]
