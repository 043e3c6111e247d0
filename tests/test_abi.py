"""CPU tests of the C ABI: the library loads, exports every declared symbol, and its
host-only functions behave; no GPU compute is called here."""
import ctypes as ct
import os
import re

import numpy as np
import pytest

from directsht_b200 import _lib as L
from oracle import dsht_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(dsht_\w+)\s*\(", src))
    return names


def test_library_built_and_loads():
    assert os.path.exists(L.LIB_PATH), "run python -m directsht_b200.build"
    lib = L.load()
    assert lib.dsht_version().decode().startswith("directsht_b200")


def test_every_declared_symbol_is_exported_and_bound():
    lib = L.load()
    declared = _declared()
    assert declared, "no declarations found"
    for name in declared:
        assert hasattr(lib, name), f"{name} not exported"
    assert declared == set(L.SIGNATURES), sorted(declared ^ set(L.SIGNATURES))


def test_index_matches_healpy_order():
    lib = L.load()
    Nl = 37
    for m in range(Nl):
        for ell in range(m, Nl):
            assert lib.dsht_index(Nl, ell, m) == O.healpy_index(ell, m, Nl)


def test_alm2cl_host_matches_oracle():
    lib = L.load()
    rng = np.random.default_rng(0)
    Nl = 20
    alm = rng.normal(size=Nl * (Nl + 1) // 2) + 1j * rng.normal(size=Nl * (Nl + 1) // 2)
    cl = np.zeros(Nl)
    L.check(lib.dsht_alm2cl(Nl, alm.view(np.float64).ctypes.data_as(ct.POINTER(ct.c_double)), L.dptr(cl)))
    np.testing.assert_allclose(cl, O.alm2cl(alm, Nl), rtol=1e-14)


def test_invalid_arguments_are_rejected_without_a_device():
    lib = L.load()
    plan = ct.c_void_p()
    assert lib.dsht_plan_create(0, 10, 0.75, 0, ct.byref(plan)) == L.DSHT_ERR_INVALID
    assert lib.dsht_plan_create(10, 1, 0.75, 0, ct.byref(plan)) == L.DSHT_ERR_INVALID
    assert lib.dsht_plan_create(10, 10, 1.5, 0, ct.byref(plan)) == L.DSHT_ERR_INVALID
    assert "invalid sizes" in L.last_error()
    assert lib.dsht_execute(None, None, None, None, 0, 0, None, None, 0, None) == L.DSHT_ERR_INVALID


def test_no_cpu_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from directsht_b200 import DirectSHT
    with pytest.raises(RuntimeError):
        DirectSHT(8, 16)
