"""The C++ FlipSim wrapper (include/ariel_flipsim.hpp) compiles against the C ABI and links
the library; without a GPU it reports ARIEL_ERR_NO_DEVICE, on a B200 it steps.

tests/cpp/integration_main.cpp is host code shaped like the reference's src/main.cpp:50-54 and
Viewer::SimLoopThread (src/viewer/viewer.cpp:66-87) with the documented edit applied: the
reference constructor's arguments (glm::vec3 dimensions, density, step size, sceneCore::Scene*,
verbose) go to ariel::FlipSim unchanged, Init seeds through the scene's own GenerateParticles and
Step's export flags reach the scene's own ExportParticles.  It builds against a stand-in Scene
with the reference's declarations (tests/cpp/reference_scene_mock.hpp)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "ariel_b200", "_lib")


def _build(tmp_path, name="flipsim_demo"):
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    exe = str(tmp_path / name)
    cmd = [cxx, "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", name + ".cpp"), "-L", LIBDIR, "-lariel_b200",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
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


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="checks the no-GPU behaviour")
def test_reference_shaped_binding_builds(tmp_path):
    r = subprocess.run([_build(tmp_path, "integration_main"), "16", "3"], capture_output=True, text=True)
    # SceneFrom read the stand-in scene (box, sphere told from other solids, gravity) before the
    # library reported that this machine has no sm_100 device
    assert "SceneFrom: liquids 1 solids 1 forces 1 box 0.350 0.500 1.000 sphere 0.6000 0.3000 0.5000 r 0.1500" \
        in r.stdout, r.stdout + r.stderr
    assert r.returncode == 3, r.stdout + r.stderr


@pytest.mark.gpu
def test_reference_shaped_binding_steps_and_exports(tmp_path):
    r = subprocess.run([_build(tmp_path, "integration_main"), "16", "3"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "frame 3 " in r.stdout and "exports 3 last export frame 3" in r.stdout and "flags 1" in r.stdout
