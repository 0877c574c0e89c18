"""The GPU's x87 extended-precision emulation (kbsrc_b200/csrc/x80.cuh) against the host's own x87 long double.

The same header compiles for the host, so the integer algorithms behind --mode ld are checked here on the CPU:
sums, differences, products and both float64 conversions, bit for bit, on 4.8 million operand pairs including
ties, cancellations, alignment shifts past the 128-bit window, denormals and the float64 subnormal boundary."""
import os
import platform
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(platform.machine().lower() not in ("x86_64", "amd64"), reason="needs x87 long double")
@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_x80_matches_host_x87(tmp_path):
    exe = tmp_path / "x80_check"
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-I", os.path.join(ROOT, "kbsrc_b200", "csrc"),
                    "-o", str(exe), os.path.join(ROOT, "tests", "x80_check.cpp")], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout
    assert r.stdout.strip().endswith("mismatches 0")
