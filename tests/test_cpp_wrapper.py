"""The C++ FlipSim wrapper (include/ariel_flipsim.hpp) compiles against the C ABI and links
the library; without a GPU it reports ARIEL_ERR_NO_DEVICE, on a B200 it steps."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "ariel_b200", "_lib")


def _build(tmp_path):
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    exe = str(tmp_path / "flipsim_demo")
    cmd = [cxx, "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "flipsim_demo.cpp"), "-L", LIBDIR, "-lariel_b200",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="checks the no-GPU behaviour")
def test_cpp_wrapper_builds_and_reports_no_device(tmp_path):
    r = subprocess.run([_build(tmp_path), "16", "1"], capture_output=True, text=True)
    assert r.returncode == 3, r.stdout + r.stderr


@pytest.mark.gpu
def test_cpp_wrapper_steps(tmp_path):
    r = subprocess.run([_build(tmp_path), "16", "3"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "frame 3 particles 7904" in r.stdout
    assert "served identical, second request 4 steps" in r.stdout
