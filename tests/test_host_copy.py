"""The staged host-transfer pipeline (orrery_b200/csrc/host_copy.cpp) on the
CPU: the unit is compiled with g++ against a host-only stand-in for the CUDA
runtime (tests/native/fake_cuda/cuda_runtime.h, whose streams run their copies
asynchronously on a thread) and ThreadSanitizer, then run: round trips of
random span lists byte for byte, injected failures raised on the calling
thread without a hang, and a working copy afterwards."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path, sanitize):
    exe = str(tmp_path / "host_copy_test")
    cmd = ["g++", "-std=c++20", "-O1", "-g", "-pthread",
           "-I", os.path.join(ROOT, "tests", "native", "fake_cuda"),
           "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "orrery_b200", "csrc"),
           os.path.join(ROOT, "tests", "native", "host_copy_test.cpp"),
           os.path.join(ROOT, "orrery_b200", "csrc", "host_copy.cpp"), "-o", exe]
    if sanitize:
        cmd[1:1] = ["-fsanitize=thread"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    return exe if res.returncode == 0 else None, res.stderr


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_staged_copy_pipeline_under_thread_sanitizer(tmp_path):
    exe, err = _build(tmp_path, sanitize=True)
    if exe is None:                      # no sanitizer runtime: the plain build still checks the bytes
        exe, err = _build(tmp_path, sanitize=False)
    assert exe is not None, err
    env = dict(os.environ, TSAN_OPTIONS="halt_on_error=1")
    res = subprocess.run([exe], capture_output=True, text=True, timeout=600, env=env)
    assert res.returncode == 0, res.stdout + res.stderr
    assert res.stdout.strip().endswith("ok")
    assert "WARNING: ThreadSanitizer" not in res.stderr
