"""CSV text of the form-factor matrix, checked on the CPU.

* The reference's own export (csv_export::export_csv,
  import_export/csv_export.cpp:26-46, committed bytes in
  tests/golden/csv_ref.npz) equals "%g" of each entry joined by ';' with '\\n'
  after each row, so "%g" of the C library is the oracle for one entry.
* The entry formatter of the CUDA kernels (form_factors_b200/csrc/ffb_csv.cuh,
  exact integer arithmetic, also valid as plain C++) equals the C library's
  "%g" on ~10 M floats: special values, every power of two, count / outgoing
  ratios, random bit patterns and whole stretches of six binades
  (tests/cpp/csv_format_check.cpp).
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
GOLDEN = os.path.join(HERE, "golden", "csv_ref.npz")

_libc = ctypes.CDLL(None)
_libc.snprintf.restype = ctypes.c_int


def c_g(x):
    """The C library's "%g" of a float widened to double."""
    buf = ctypes.create_string_buffer(64)
    _libc.snprintf(buf, 64, b"%g", ctypes.c_double(float(x)))
    return buf.value


def test_reference_export_is_percent_g_of_each_entry():
    g = np.load(GOLDEN)
    ff, text = g["ff"], g["text"].tobytes()
    rows = [b";".join(c_g(v) for v in row) + b"\n" for row in ff]
    assert b"".join(rows) == text


def test_golden_matrix_covers_every_form():
    text = np.load(GOLDEN)["text"].tobytes()
    for token in (b"-0;", b"inf", b"-inf", b"nan", b"-nan", b"e+38", b"e-45", b"0.0001", b"e-05", b"1e+06",
                  b"100000;"):
        assert token in text, token


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_entry_formatter_matches_c_library(tmp_path):
    exe = str(tmp_path / "csv_format_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "form_factors_b200", "csrc"), "-o", exe,
                    os.path.join(HERE, "cpp", "csv_format_check.cpp")], check=True)
    r = subprocess.run([exe, "1000000", "7"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches 0" in r.stdout
