"""The multiply-high division of the stencil kernels' index decompositions
(cubismnova_b200/csrc/cn_fastdiv.h), host path, against exact division:
compiled with the host compiler, no GPU needed."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_fastdiv_matches_integer_division(tmp_path):
    exe = str(tmp_path / "fastdiv_test")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "cubismnova_b200", "csrc"),
                    "-I", "/usr/local/cuda/include", os.path.join(ROOT, "tests", "cpp", "fastdiv_test.cpp"),
                    "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
