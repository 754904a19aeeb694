"""Bitsliced GF(16) helpers of the CUDA engine, compiled as host code and run on the CPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bitsliced_helpers_on_host(tmp_path):
    from cumayo_b200.build import nvcc
    try:
        cc = nvcc()
    except RuntimeError:
        pytest.skip("nvcc not available")
    exe = tmp_path / "host_arith"
    r = subprocess.run([cc, "-std=c++17", "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "cumayo_b200", "csrc"),
                        "-o", str(exe), os.path.join(ROOT, "tests", "host_arith_test.cu")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.stdout.strip() == "OK", out.stdout
