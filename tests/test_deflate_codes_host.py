"""The compressor's code construction (cubam_b200/csrc/deflate_codes.cuh) checked on the host.

tests/deflate_codes_check.cu is built with nvcc as a host program (no GPU) and run: the
count-based code lengths the kernel computes equal the serial minimum-redundancy lengths, every
code is complete and within its limit, per-run coding of code lengths equals whole-sequence coding
and expands back, and the length/distance symbols agree with RFC 1951's tables.
"""

import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


def test_code_construction_on_the_host(tmp_path):
    from cubam_b200 import build

    try:
        nvcc = build.nvcc()
    except RuntimeError:
        pytest.skip("nvcc not found")
    exe = tmp_path / "deflate_codes_check"
    subprocess.run([nvcc, "-O2", "-std=c++17", "-Wno-deprecated-gpu-targets", str(HERE / "deflate_codes_check.cu"),
                    "-o", str(exe)], check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("0 failures")
