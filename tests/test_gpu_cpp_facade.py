"""The C++ facade (include/cubismnova_b200.hpp): compile a program with the
host compiler against the C ABI library and run the reference's BC/FieldLab
assertions on the GPU, and an HDF5 write / read of a grid (in a scratch
directory)."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_facade_reference_assertions(cn, tmp_path):
    libdir = os.path.join(ROOT, "cubismnova_b200")
    exe = str(tmp_path / "facade_test")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "facade_test.cpp"), "-L", libdir, "-lcubismnova_b200",
                    "-Wl,-rpath," + libdir, "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120, cwd=str(tmp_path))
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
