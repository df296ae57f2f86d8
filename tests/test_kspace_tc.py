"""GPU: the k-space force of the mixed form on the tensor cores.

k_kforce_tc contracts each atom's phases z_m with the force coefficients of
every (nx, ny) column on tcgen05 (TF32 hi/lo split operands: FP32-level
sums) and must give the CUDA-core kernel's force and, through it, the
reference's.  Checked through the C ABI:
  * the 500-ion reference fixture (kmax 4) and the 8000-ion benchmark system
    (kmax 8, 289 columns in five tiles over a two-block cluster): total
    accelerations within 1e-7 (global relative) / 2e-6 (max over rms) of
    the CUDA-core kernel's, and within the usual 1e-5 of the reference's;
  * a 40-step run with list rebuilds stays within 1e-6 of the CUDA-core run;
  * k_max beyond what the tensor-core tile holds (k_max 30) falls back to
    the CUDA-core kernel (same forces bit for bit under either setting);
  * a non-cubic box with per-axis k_max (5, 3, 4), whose truncated k-set
    leaves some (nx, ny) columns without their mirror: forces and S(k) of
    both precisions against the FP64 oracle (the S(k) sums and the force
    use one column of each mirror pair).
"""
import numpy as np
import pytest

from helpers import force_errors, load_ref_fixture

pytestmark = pytest.mark.gpu


def forces(abi, s, kind, steps=0):
    sim = abi.Simulation(s, precision=abi.PREC_MIXED)
    sim.set_kspace_force_kernel(kind)
    if steps:
        sim.run(steps)
        pos, vel, acc = sim.state()
        sim.close()
        return pos, vel, acc
    acc, _ = sim.compute_forces()
    sim.close()
    return acc


@pytest.mark.parametrize("name", ["ions500", "ions8000"])
def test_tensor_core_kforce_matches_cuda_cores(cuda_lib, name):
    from caviar_b200 import workloads as W
    if name == "ions500":
        s, d = load_ref_fixture("ions500")
    else:
        s, d = W.config_ions_8000(), None
    tc = forces(cuda_lib, s, cuda_lib.KFORCE_AUTO)
    cc = forces(cuda_lib, s, cuda_lib.KFORCE_CUDA_CORES)
    assert np.isfinite(tc).all()
    g, mx, _ = force_errors(tc, cc)
    print(f"{name}: tensor cores vs CUDA cores: global {g:.2e}, max/rms {mx:.2e}")
    assert g <= 1e-7 and mx <= 2e-6, (g, mx)
    if d is not None:
        g, mx, _ = force_errors(tc, d["ref_acc"].reshape(-1, 3))
        assert g <= 1e-5 and mx <= 1e-5, (g, mx)


def test_tensor_core_kforce_trajectory(cuda_lib):
    from caviar_b200 import workloads as W
    s = W.random_ions(1000, 20.0, seed=4, rc=6.0, kmax=6, alpha=0.5)
    p1, v1, _ = forces(cuda_lib, s, cuda_lib.KFORCE_AUTO, steps=40)
    p2, v2, _ = forces(cuda_lib, s, cuda_lib.KFORCE_CUDA_CORES, steps=40)
    dp = p1 - p2
    dp -= s.box * np.round(dp / s.box)
    print(f"40 steps: max |dr| {np.abs(dp).max():.2e}, max |dv| {np.abs(v1 - v2).max():.2e}")
    assert np.abs(dp).max() < 1e-6 and np.abs(v1 - v2).max() < 1e-4


def test_large_kmax_uses_cuda_cores(cuda_lib):
    from caviar_b200 import workloads as W
    s = W.random_ions(100, 12.0, seed=9, rc=5.0, kmax=30, alpha=0.8)
    a = forces(cuda_lib, s, cuda_lib.KFORCE_AUTO)
    b = forces(cuda_lib, s, cuda_lib.KFORCE_CUDA_CORES)
    assert np.array_equal(a, b)


def _anisotropic_system():
    from caviar_b200 import workloads as W
    s = W.random_ions(600, 16.0, seed=21, rc=6.0, kmax=4, alpha=0.6)
    scale = np.array([1.0, 1.1, 1.2])  # expanded only: the generator's minimum separation holds
    s.pos = s.lo + (s.pos - s.lo) * scale
    s.hi = s.lo + (s.hi - s.lo) * scale
    s.ewald_k = W.EwaldKParams(alpha=0.6, kmax=(5, 3, 4), k_electrostatic=s.ewald_k.k_electrostatic)
    return s


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_anisotropic_kmax_noncubic_box_vs_oracle(cuda_lib, oracle_lib, prec):
    s = _anisotropic_system()
    o = oracle_lib.Oracle(s)
    o.setup()
    ref_acc, ref_sk = o.state()[2], o.sk()
    p = cuda_lib.PREC_FP64 if prec == "fp64" else cuda_lib.PREC_MIXED
    sim = cuda_lib.Simulation(s, precision=p)
    acc, th = sim.compute_forces()
    sk = sim.sk()
    if prec == "mixed":
        assert sim.info()["kspace_tensor_cores"] == 1
    sim.close()
    g, mx, _ = force_errors(acc, ref_acc)
    dsk = np.abs(sk - ref_sk).max() / np.abs(ref_sk).max()
    print(f"{prec}: forces global {g:.2e}, max/rms {mx:.2e}; S(k) {dsk:.2e}")
    tol = 1e-11 if prec == "fp64" else 1e-5
    assert len(sk) == len(ref_sk) == 480
    assert g <= tol and mx <= (1e-10 if prec == "fp64" else 1e-5), (g, mx)
    assert dsk <= tol, dsk
