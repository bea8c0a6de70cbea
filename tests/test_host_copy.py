"""The threaded host copies of libvoss (parallel_copy, parallel_gather: the request server's
candidate payloads and the staged transfers) on the CPU: tests/host_copy_check.cpp is linked
against the library's object files, which the build leaves in voss-prime-gaps_v1_b200/_build."""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(os.path.dirname(HERE), "voss-prime-gaps_v1_b200")
NVCC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
OBJS = ["sieve_kernels", "mr_kernels", "voss_api", "voss_artifacts", "voss_server", "voss_driver",
        "cert_kernels", "large_sort", "short_iv"]


def test_parallel_copy_and_gather_equal_plain_concatenation(tmp_path):
    objs = [os.path.join(PKG, "_build", o + ".o") for o in OBJS]
    if not all(os.path.exists(o) for o in objs) or not os.path.exists(NVCC):
        pytest.skip("library objects or nvcc not present (run the build first)")
    exe = str(tmp_path / "host_copy_check")
    subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17",
                    "-I", os.path.join(os.path.dirname(HERE), "include"), "-I", os.path.join(PKG, "csrc"),
                    "-o", exe, os.path.join(HERE, "host_copy_check.cpp")] + objs, check=True, timeout=600)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "bad=0" in r.stdout, r.stdout + r.stderr
