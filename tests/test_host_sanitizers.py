"""The host half of the library (formats, CSR builder and validator,
generators) under AddressSanitizer and UndefinedBehaviorSanitizer: tests/host_fuzz.cpp
feeds it corrupted files and random arrays, and any sanitizer report fails
the test.  Needs g++ only (no GPU, no CUDA runtime calls)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "dyn_maxflow_b200", "csrc")


def _cuda_include():
    for d in (os.environ.get("CUDA_HOME"), "/usr/local/cuda"):
        if d and os.path.exists(os.path.join(d, "include", "cuda_runtime.h")):
            return os.path.join(d, "include")
    return None


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_host_code_is_clean_under_sanitizers(tmp_path, golden_dir):
    exe = str(tmp_path / "host_fuzz")
    cmd = ["g++", "-std=c++17", "-O1", "-g", "-fopenmp", "-fsanitize=address,undefined", "-fno-omit-frame-pointer",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    inc = _cuda_include()
    if inc:
        cmd += ["-I", inc]
    cmd += [os.path.join(ROOT, "tests", "host_fuzz.cpp"), os.path.join(CSRC, "dmf_host.cpp"), "-o", exe]
    b = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    if b.returncode != 0 and "sanitizer" in b.stderr.lower() and "cannot find" in b.stderr.lower():
        pytest.skip("sanitizer runtime not installed")
    assert b.returncode == 0, b.stderr[-3000:]
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1:halt_on_error=1", OMP_NUM_THREADS="4")
    r = subprocess.run([exe, os.path.join(golden_dir, "johnson8-2-4.bin"), os.path.join(golden_dir, "johnson_p1.bin"),
                        str(tmp_path / "scratch.bin"), "2000"], capture_output=True, text=True, timeout=600, env=env)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out[-3000:]
    assert "runtime error" not in out and "AddressSanitizer" not in out and "LeakSanitizer" not in out, out[-3000:]
    assert "generators: edge parameters done" in r.stdout
