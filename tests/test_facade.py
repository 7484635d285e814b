"""The C++ facade (include/hila_b200/wilson.hpp): it compiles against the C ABI
(CPU), and the reference's test program written against it passes on the GPU:
tests/cpp/test_cg_facade.cpp (the Dirac_Wilson_evenodd block with a GaugeField)
and tests/cpp/test_cg_reference_blocks.cpp (the Dirac_Wilson, staggered,
Dirac_Wilson_evenodd and Hasenbusch blocks of test_CG.cpp:127-353 written as a
HILA application writes them: Field<SU<3,double>> U[4], boundary conditions set
per field, MRE_guess)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_cg_facade.cpp")
BLOCKS = os.path.join(ROOT, "tests", "cpp", "test_cg_reference_blocks.cpp")
LIBDIR = os.path.join(ROOT, "hila_b200")


def _cxx():
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def build(tmp_path, src=SRC):
    exe = str(tmp_path / os.path.splitext(os.path.basename(src))[0])
    cmd = [_cxx(), "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), src, "-o", exe,
           "-L", LIBDIR, "-lhila_b200", f"-Wl,-rpath,{LIBDIR}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return exe


def test_facade_compiles(hw, tmp_path):
    if not os.path.exists(hw.LIB_PATH):
        from hila_b200 import build as hb
        hb.build()
    assert os.path.exists(build(tmp_path))
    assert os.path.exists(build(tmp_path, BLOCKS))


@pytest.mark.gpu
def test_facade_reference_cg_test(hw, ctx, tmp_path):
    exe = build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "facade test passed" in r.stdout


@pytest.mark.gpu
def test_facade_reference_blocks(hw, ctx, tmp_path):
    exe = build(tmp_path, BLOCKS)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "reference blocks passed" in r.stdout
