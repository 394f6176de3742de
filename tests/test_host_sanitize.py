"""Host-side code of the library under AddressSanitizer and
UndefinedBehaviorSanitizer: tests/host_sanitize.cpp drives the JSON
configuration reader (csrc/json.hpp) and the PlaneImpactResponse build
(csrc/pir.cpp), compiled with -fsanitize=address,undefined.  CPU only."""

import os
import shutil
import subprocess

import pytest

from conftest import ROOT

CSRC = os.path.join(ROOT, "wire-cell-toolkit_b200", "csrc")


def test_host_code_under_asan_ubsan(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "host_sanitize")
    cmd = ["g++", "-std=c++17", "-O1", "-g", "-fno-omit-frame-pointer", "-fsanitize=address,undefined",
           "-fno-sanitize-recover=all", "-Wall", "-Werror", "-I", CSRC,
           os.path.join(ROOT, "tests", "host_sanitize.cpp"), os.path.join(CSRC, "pir.cpp"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1", UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([exe], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
