"""The C++ system types (include/ffb_systems.h) through the reference's own
interfaces: the test program tests/cpp/test_systems.cpp, built standalone
against this repository's headers, and -- where the reference build exists --
against the reference's headers and objects (oracle/_ref/test_systems_ref),
where the reference's casters, emitter and calculator run beside and mixed
with the B200 types."""
import os
import subprocess

import pytest

from form_factors_b200 import build

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(exe, cwd):
    # cwd: the program writes (and removes) its CSV files there
    p = subprocess.run([exe], capture_output=True, text=True, timeout=600, cwd=str(cwd))
    assert p.returncode == 0, p.stdout + p.stderr[-4000:]
    return p.stdout


def test_systems_standalone(tmp_path):
    build.build()
    exe = str(tmp_path / "test_systems")
    subprocess.run(["g++", "-std=c++11", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "test_systems.cpp"), "-L", build.PKG, "-lffb200",
                    "-Wl,-rpath," + build.PKG, "-o", exe], check=True)
    out = _run(exe, tmp_path)
    assert " 0 failures" in out


def test_systems_with_reference(tmp_path):
    exe = os.path.join(ROOT, "oracle", "_ref", "test_systems_ref")
    if not os.path.exists(exe):
        pytest.skip("reference build of the system test not present (make -C oracle systest)")
    out = _run(exe, tmp_path)
    assert " 0 failures" in out
