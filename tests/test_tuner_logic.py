"""The launch-shape tuner's decision logic (hila_b200/csrc/engine_tune.h) on the CPU:
tests/cpp/test_tuner.cpp feeds it made-up chunk timings and checks which candidate
each chunk runs, what counts as a sample, and when a work class is decided."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_tuner.cpp")


def test_tuner_logic(tmp_path):
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    exe = str(tmp_path / "test_tuner")
    subprocess.run([cxx, "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "hila_b200", "csrc"),
                    SRC, "-o", exe], check=True, capture_output=True, text=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "tuner logic passed" in r.stdout
