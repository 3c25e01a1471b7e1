"""The C++ drop-in header compiles into a ParlayANN-style program (CPU), and
that program builds, saves, reloads and searches an index on the GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def compile_demo(out):
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "dropin_demo.cpp"), "-o", out,
           "-L", os.path.join(ROOT, "parlayann_b200"), "-lparlayann_b200",
           "-Wl,-rpath," + os.path.join(ROOT, "parlayann_b200")]
    subprocess.run(cmd, check=True, capture_output=True)


def test_dropin_header_compiles_and_links(tmp_path, lib_built):
    out = str(tmp_path / "dropin_demo")
    compile_demo(out)
    assert os.path.exists(out)


@pytest.mark.gpu
def test_dropin_program_runs_on_gpu(tmp_path, lib_built):
    out = str(tmp_path / "dropin_demo")
    compile_demo(out)
    r = subprocess.run([out, str(tmp_path / "g.bin")], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "beam_search agrees 1" in r.stdout
