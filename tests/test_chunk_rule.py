"""The pressure solve's per-scene chunk rule (ariel_b200/csrc/pcg.cuh) never needs more
partial-sum slots than the layout reserves for a scene of that size: the solve writes one slot
per chunk, so a count above the bound would write past the array.  The rule's host/device
functions are compiled into a small host program and checked over every FLUID count of grids up
to 96^3 and sampled counts of grids up to 1024^3; no GPU is needed."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_chunk_bound_covers_every_fluid_count(tmp_path):
    from ariel_b200 import build as B
    exe = str(tmp_path / "chunk_rule")
    cmd = [B.nvcc()] + B.ARCH + ["-std=c++17", "-O2", "-ccbin", B.host_compiler(),
                                 "-I", os.path.join(ROOT, "ariel_b200", "csrc"),
                                 os.path.join(ROOT, "tests", "cpp", "chunk_rule.cu"), "-o", exe]
    subprocess.run(cmd, check=True, capture_output=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
