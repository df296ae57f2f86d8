"""CPU: the C-ABI library builds, loads, and exports every symbol that
include/caviar_b200.h declares; without a GPU it fails loudly (no CPU path)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "caviar_b200.h")) as f:
        src = f.read()
    return sorted(set(re.findall(r"\b(cvr_[a-z_]+)\s*\(", src)))


def test_header_and_binding_agree(cuda_lib):
    assert declared_symbols() == sorted(cuda_lib.EXPORTED)


def test_library_exports_every_declared_symbol(cuda_lib):
    lib = ctypes.CDLL(cuda_lib.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_no_cpu_fallback_without_gpu(cuda_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from caviar_b200 import workloads as W
    s = W.fcc_lattice(3, 0.8442, 0.72, seed=1)
    with pytest.raises(cuda_lib.CvrError):
        cuda_lib.Simulation(s)


def test_invalid_arguments_rejected(cuda_lib):
    L = cuda_lib.load()
    h = ctypes.c_void_p()
    import numpy as np
    lo = np.zeros(3)
    hi = np.zeros(3)  # hi <= lo
    bc = (ctypes.c_int * 3)(1, 1, 1)
    m = np.ones(1)
    rc = L.cvr_create(ctypes.byref(h), lo.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                      hi.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), bc, 1,
                      m.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None, 0)
    assert rc == 1 and not h.value
