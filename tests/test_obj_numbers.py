"""The OBJ number conversions of the GPU importer (form_factors_b200/csrc/
ffb_obj.cuh, built as plain C++) against the C library that the reference's
importer calls through sscanf (import_export/obj_import.cpp:193-224): "%f"
(strtof: correctly rounded, ties to even; exact midpoints written with 40
digits, hexadecimal floats, subnormals, infinities, NaNs, scanf's own
consumption rules) and the three face formats (tests/cpp/obj_number_check.cpp)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_obj_numbers_match_c_library(tmp_path):
    exe = str(tmp_path / "obj_number_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "form_factors_b200", "csrc"), "-o", exe,
                    os.path.join(HERE, "cpp", "obj_number_check.cpp")], check=True)
    r = subprocess.run([exe, "200000", "11"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches 0" in r.stdout
