"""The host half of the library (formats, CSR builder and validator,
generators) and the dmf_tool command line under AddressSanitizer and
UndefinedBehaviorSanitizer: tests/host_fuzz.cpp feeds the library corrupted
files and random arrays, and the tool gets malformed text files and bad
arguments; any sanitizer report fails the test.  Needs g++ only (no GPU, no
CUDA runtime calls)."""
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


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_tool_text_commands_are_clean_under_sanitizers(tmp_path, golden_dir):
    """dmf_tool's text commands (weight, cb, cb_update) and generator argument
    checks on malformed inputs: every run ends with a status and no
    sanitizer report."""
    import random
    exe = str(tmp_path / "dmf_tool_san")
    cmd = ["g++", "-std=c++17", "-O1", "-g", "-fopenmp", "-fsanitize=address,undefined", "-fno-omit-frame-pointer",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC]
    inc = _cuda_include()
    if inc:
        cmd += ["-I", inc]
    cmd += [os.path.join(CSRC, "dmf_tool.cpp"), os.path.join(CSRC, "dmf_host.cpp"), "-o", exe]
    b = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert b.returncode == 0, b.stderr[-3000:]
    rng = random.Random(3)
    lines = open(os.path.join(golden_dir, "johnson8-2-4.txt")).read().splitlines()
    odd = ["", "%", "% comment", "1", "1 2", "a b c", "-1 2 5", "2147483647 1 1", "1 2 99999999999", "3 3 3",
           "0 0", "1 2 3 4 5 6", "9999999 1 2"]
    inputs = [x + "\n" for x in odd]
    for _ in range(27):
        ls = lines[:rng.randint(0, len(lines))]
        for _ in range(rng.randint(0, 4)):
            ls.insert(rng.randint(0, len(ls)), rng.choice(odd))
        inputs.append("\n".join(ls) + ("\n" if rng.random() < 0.5 else ""))
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1", UBSAN_OPTIONS="print_stacktrace=1", OMP_NUM_THREADS="2")
    src, out = str(tmp_path / "in.txt"), str(tmp_path / "out.bin")
    runs = [[c, src, out] for c in ("weight", "cb", "cb_update")]
    graph = os.path.join(golden_dir, "johnson8-2-4.bin")
    bad_args = [["gen-grid", "0", "0", "1", out], ["gen-grid", "x", "3", "1", out], ["gen-rmat", "40", "1", "0", out],
                ["gen-rmat", "4", "1", "-5", out], ["gen-batches", graph, "-3", "0.1", "1", str(tmp_path / "b")],
                ["gen-batches", graph, "3", "7", "1", str(tmp_path / "b")],
                ["gen-grid", "4", "4", "1", str(tmp_path / "missing" / "g.bin")], ["bogus"], []]
    for text in inputs:
        with open(src, "w") as f:
            f.write(text)
        for args in runs:
            r = subprocess.run([exe] + args, capture_output=True, text=True, timeout=120, env=env)
            log = r.stdout + r.stderr
            assert r.returncode in (0, 1), (args[0], text[:200], log[-2000:])
            assert "runtime error" not in log and "Sanitizer" not in log, (args[0], text[:200], log[-2000:])
    for args in bad_args:
        r = subprocess.run([exe] + args, capture_output=True, text=True, timeout=120, env=env)
        log = r.stdout + r.stderr
        assert r.returncode in (1, 2), (args, log[-2000:])
        assert "runtime error" not in log and "Sanitizer" not in log, (args, log[-2000:])
