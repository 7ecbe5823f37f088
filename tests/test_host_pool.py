"""CPU stress check of the host worker pool that runs the library's parallel
host passes (packing, validation, readback): concurrent callers and passes
nested inside a chunk, at several host thread counts, against serial sums.
The check is a small host program built with nvcc from tests/native/."""

import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not available")
def test_pool_runs_concurrent_and_nested_passes(tmp_path):
    exe = str(tmp_path / "pool_check")
    subprocess.run(["nvcc", "-Wno-deprecated-gpu-targets", "-std=c++17", "-O2", "-x", "cu", os.path.join(HERE, "native", "pool_check.cu"),
                    "-o", exe, "-lpthread"], check=True, timeout=600)
    for threads in ("1", "3", "16"):
        r = subprocess.run([exe], env=dict(os.environ, TMPM_HOST_THREADS=threads), capture_output=True, text=True,
                           timeout=120)
        assert r.returncode == 0 and r.stdout.strip() == "OK", (threads, r.stdout, r.stderr)
