"""The C-ABI library: loads, exports every declared entry point, and its
host-only logic behaves like the reference (CPU only; no compute calls)."""
import ctypes as C
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b(cn_[a-z0-9_]+|field[A-Za-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_all_declared_symbols():
    from cubismnova_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build()
    lib = C.CDLL(_lib.LIB_PATH)
    names = declared_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_abi_version_and_status_strings():
    from cubismnova_b200 import _lib
    lib = _lib.lib()
    assert lib.cn_abi_version() == 1
    assert lib.cn_status_string(2).decode() == "Stencil: begin_ must be <= 0"
    assert lib.cn_status_string(3).decode() == "Stencil: end_ must be > 0"
    assert lib.cn_status_string(6).decode() == "FieldLab: no field loaded"
    assert lib.cn_status_string(5).decode() == \
        "FieldLab: can not load lab data when not allocated first"


def test_stencil_checks_like_reference():
    """Core/StencilTest.cpp:12-51 plus the all-components comparison rule."""
    from cubismnova_b200 import Core
    s0 = Core.Stencil(-2, 3)
    assert s0.getBegin() == (-2, -2, -2) and s0.getEnd() == (3, 3, 3)
    assert not s0.isTensorial()
    s1 = Core.Stencil((-6,) * 3, (3,) * 3, True)
    assert s1.isTensorial()
    with pytest.raises(RuntimeError, match=r"^Stencil: end_ must be > 0$"):
        Core.Stencil(0, 0)
    with pytest.raises(RuntimeError, match=r"^Stencil: begin_ must be <= 0$"):
        Core.Stencil(1, 4)
    # the reference accepts a single violating component; the device lab
    # cannot represent it and rejects it with its own message
    with pytest.raises(RuntimeError, match="every dimension"):
        Core.Stencil((1, 0, 0), (2, 2, 2))


def test_bc_descriptors():
    from cubismnova_b200 import BC
    assert BC.Dirichlet(0, 0, 10).name() == "Dirichlet"
    assert BC.Absorbing(1, 1).name() == "Zeroth-Order Absorbing"
    assert BC.Symmetry(2, 0).name() == "Symmetry"
    d = BC.Dirichlet(0, 0, 10)
    assert d.getValue() == 10
    info = BC.Absorbing(1, 1).getBoundaryInfo()
    assert (info.dir, info.side, info.is_periodic) == (1, 1, False)
    assert BC.Base(2, 0).getBoundaryInfo().is_periodic


def test_no_gpu_fails_loudly():
    """Without a usable GPU the product raises; it never computes on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from cubismnova_b200 import Grid
    with pytest.raises(RuntimeError, match="CUDA"):
        Grid.Cartesian(2, 4)


def test_product_does_not_import_oracle():
    """The product package never reaches into the test oracle."""
    for p in glob.glob(os.path.join(ROOT, "cubismnova_b200", "**", "*.py"), recursive=True):
        src = open(p).read()
        assert not re.search(r"^\s*(import|from)\s+oracle\b", src, flags=re.M), p
    for p in glob.glob(os.path.join(ROOT, "cubismnova_b200", "csrc", "*")):
        assert "cn_oracle" not in open(p).read(), p


def test_cpp_facade_compiles():
    """The C++ facade compiles with the host compiler (no GPU needed)."""
    import subprocess
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"),
                            os.path.join(ROOT, "tests", "cpp", "facade_test.cpp")],
                           capture_output=True, text=True, cwd=d)
        assert r.returncode == 0, r.stderr
