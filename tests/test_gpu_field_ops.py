"""The FieldOperator.h:149-227 hooks (fieldAdd2_double, ..., fieldRcp_float)
on device and host pointers, bit-exact against the loops of
Block/FieldOperator.h:16-30 restated in numpy (IEEE, no contraction)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OPS = [("Add", np.add), ("Sub", np.subtract), ("Mul", np.multiply), ("Div", np.divide)]


@pytest.mark.parametrize("dtype,suffix,ct", [(np.float64, "double", C.c_double), (np.float32, "float", C.c_float)])
@pytest.mark.parametrize("where", ["device", "host"])
def test_field_hooks(cn, dtype, suffix, ct, where):
    import torch
    lib = cn._lib.lib()
    rng = np.random.default_rng(1)
    n = 100003
    a = (rng.standard_normal(n) + 3).astype(dtype)
    b = (rng.standard_normal(n) + 3).astype(dtype)
    s = dtype(1.7)
    if where == "device":
        ta, tb, td = torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), torch.empty(n, dtype=torch.from_numpy(a).dtype, device="cuda")
        pa, pb, pd = C.c_void_p(ta.data_ptr()), C.c_void_p(tb.data_ptr()), C.c_void_p(td.data_ptr())
        get = lambda: td.cpu().numpy()
    else:
        d = np.empty_like(a)
        pa, pb, pd = a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p), d.ctypes.data_as(C.c_void_p)
        get = lambda: d.copy()
    for name, f in OPS:
        fn2 = getattr(lib, f"field{name}2_{suffix}")
        fn2.restype = None
        fn2.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]
        fn2(pa, pb, pd, n)
        assert np.array_equal(get(), f(a, b)), name + "2"
        fn1 = getattr(lib, f"field{name}1_{suffix}")
        fn1.restype = None
        fn1.argtypes = [C.c_void_p, ct, C.c_void_p, C.c_size_t]
        fn1(pa, ct(s), pd, n)
        assert np.array_equal(get(), f(a, s)), name + "1"
    fr = getattr(lib, f"fieldRcp_{suffix}")
    fr.restype = None
    fr.argtypes = [C.c_void_p, ct, C.c_void_p, C.c_size_t]
    fr(pa, ct(s), pd, n)
    assert np.array_equal(get(), s * (dtype(1) / a))
