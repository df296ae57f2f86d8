"""GPU: the allocation-free structure-factor entry point.

cvr_structure_factor_noalloc serves callers that cannot allocate device
memory: code inside a host program whose allocator owns the GPU's memory, a
plug-in that may not allocate after start-up, or a caller that cannot take
the device-wide synchronisation of cudaMalloc/cudaFree mid-run.  The caller
brings the input and output buffers (here: tensors the test allocates); the
entry point keeps its partial sums in one fixed device array.

Checked through the C ABI against the regular path (cvr_compute_forces +
cvr_get_sk, FP64 form) with the FP64 S(k) tolerance of the parity tests
(1e-11 of max |S|), on two calls in a row, with a call of a different size in
between to show that leftovers in the shared array do not leak into results.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from helpers import ewald_golden, load_ref_fixture

pytestmark = pytest.mark.gpu


def _entry(abi):
    f = abi.load().cvr_structure_factor_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                  ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    f.restype = ctypes.c_int
    return f


def _regular_sk(abi, s):
    sim = abi.Simulation(s, precision=abi.PREC_FP64)
    sim.compute_forces()
    sk = sim.sk()
    sim.close()
    return sk


def _noalloc_sk(abi, torch, f, s):
    pos = torch.tensor(np.ascontiguousarray(s.pos), dtype=torch.float64, device="cuda")
    q = torch.tensor(np.asarray(s.charge)[s.type], dtype=torch.float64, device="cuda")
    kx, ky, kz = s.ewald_k.kmax
    nk = 8 * kx * ky * kz
    out = torch.full((nk, 2), float("nan"), dtype=torch.float64, device="cuda")
    box = (ctypes.c_double * 3)(*[float(x) for x in s.box])
    err = ctypes.create_string_buffer(256)
    rc = f(pos.data_ptr(), q.data_ptr(), s.n, box, kx, ky, kz, out.data_ptr(),
           ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), err, 256)
    assert rc == 0, err.value.decode()
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    return o[:, 0] + 1j * o[:, 1]


def test_noalloc_structure_factor_matches_regular_path(cuda_lib):
    import torch
    f = _entry(cuda_lib)
    s, d = load_ref_fixture("ions500")
    ref = _regular_sk(cuda_lib, s)
    assert np.isfinite(ref).all() and len(ref) == 8 * 4 ** 3
    tol = 1e-11 * np.abs(ref).max()
    first = _noalloc_sk(cuda_lib, torch, f, s)
    assert np.abs(first - ref).max() <= tol
    # a larger call in between (kmax 30: 216000 k-vectors) overwrites the shared array
    g, _, _ = ewald_golden()
    big_ref = _regular_sk(cuda_lib, g)
    big = _noalloc_sk(cuda_lib, torch, f, g)
    assert np.abs(big - big_ref).max() <= 1e-11 * np.abs(big_ref).max()
    second = _noalloc_sk(cuda_lib, torch, f, s)
    assert np.abs(second - ref).max() <= tol
    # and it agrees with the reference's own S(k) for this state
    ref_sk = d["ref_sk"][0::2] + 1j * d["ref_sk"][1::2]
    assert np.abs(second - ref_sk).max() <= tol


def test_noalloc_rejects_sizes_beyond_the_maximum(cuda_lib):
    import torch
    f = _entry(cuda_lib)
    box = (ctypes.c_double * 3)(10.0, 10.0, 10.0)
    err = ctypes.create_string_buffer(256)
    # real device buffers of the stated sizes, so that nothing could read
    # through a bad address even if a check came after a launch
    pos = torch.zeros((100, 3), dtype=torch.float64, device="cuda")
    q = torch.zeros(100, dtype=torch.float64, device="cuda")
    out = torch.zeros((8, 2), dtype=torch.float64, device="cuda")
    rc = f(pos.data_ptr(), q.data_ptr(), 100, box, 31, 31, 31, out.data_ptr(), None, err, 256)
    assert rc == 1 and b"k_max" in err.value
    rc = f(pos.data_ptr(), q.data_ptr(), 0, box, 1, 1, 1, out.data_ptr(), None, err, 256)
    assert rc == 1
    torch.cuda.synchronize()
    assert not out.any()
