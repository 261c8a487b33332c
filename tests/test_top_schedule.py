"""Top-region chunk schedule checked on the host (tests/top_schedule_check.cpp):
block chunks and warp rounds never read a score they write, warp chunks are
whole rounds within a buffer, and the schedule gives the level-by-level
sweep result, for several region and chunk sizes (down to one 32-edge
round per buffer)."""
import os
import subprocess

from conftest import ROOT

HERE = os.path.dirname(os.path.abspath(__file__))


def test_top_schedule_matches_level_order(tmp_path):
    exe = str(tmp_path / "top_schedule_check")
    lib = os.path.join(ROOT, "chsga_b200", "lib")
    subprocess.run(["g++", "-O2", "-std=c++17", "-fopenmp",
                    "-I", os.path.join(ROOT, "chsga_b200", "csrc"), "-I", os.path.join(ROOT, "include"),
                    "-o", exe, os.path.join(HERE, "top_schedule_check.cpp"),
                    os.path.join(ROOT, "chsga_b200", "csrc", "device_graph.cpp"),
                    "-L", lib, "-lchsga", "-Wl,-rpath," + lib], check=True, timeout=300)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.startswith("OK")
