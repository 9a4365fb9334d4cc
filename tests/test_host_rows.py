"""Host expansion of packed count blocks (ffb_host_rows.cpp), on the CPU.

A count matrix written to a host buffer crosses PCIe as the (column, count)
pairs of each row block's nonzero entries; host threads write the dense rows
from them.  tests/cpp/host_rows_check.cpp builds that code standalone with
g++ and compares it with a plain dense construction over random row widths,
densities, destination alignments and thread counts.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not found")
def test_host_row_expansion(tmp_path):
    exe = str(tmp_path / "host_rows_check")
    csrc = os.path.join(ROOT, "form_factors_b200", "csrc")
    subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-I", os.path.join(ROOT, "include"), "-I", csrc,
                    os.path.join(ROOT, "tests", "cpp", "host_rows_check.cpp"), os.path.join(csrc, "ffb_host_rows.cpp"),
                    "-o", exe], check=True)
    p = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.startswith("OK")
