"""The library's host-side coders under AddressSanitizer and
UndefinedBehaviorSanitizer: tests/fuzz_host.cpp, built here from their sources
(csrc/intra.cpp, csrc/jbig.cpp), feeds them random and damaged inputs, each in
a heap block of exactly its size (intra decoder: random bit strings; intra
encoder: random frames, decoded back; JBIG decoder: cut or bit-flipped
streams and random bytes)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "dvc_b200", "csrc")


@pytest.fixture(scope="module")
def fuzz_bin(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    out = str(tmp_path_factory.mktemp("fuzz") / "fuzz_host")
    cmd = [gxx, "-O1", "-g", "-std=c++17", "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
           "-fno-omit-frame-pointer", "-I", os.path.join(ROOT, "include"), "-o", out,
           os.path.join(ROOT, "tests", "fuzz_host.cpp"), os.path.join(CSRC, "intra.cpp"), os.path.join(CSRC, "jbig.cpp")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0 and "sanitize" in r.stderr:
        pytest.skip("sanitizer runtime not available: " + r.stderr[-200:])
    assert r.returncode == 0, r.stderr[-2000:]
    return out


@pytest.mark.parametrize("mode,iters", [("intra_dec", 6000), ("intra_enc", 150), ("jbig_dec", 12000)])
def test_host_coders_under_sanitizers(fuzz_bin, mode, iters):
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=0:abort_on_error=1", UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([fuzz_bin, mode, str(iters)], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0 and "runtime error" not in r.stderr and "Sanitizer" not in r.stderr, r.stderr[-3000:]
