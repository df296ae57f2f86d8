"""GPU parity at the benchmark systems themselves (through the C ABI).

The systems are the seeded generators the bench times
(caviar_b200.workloads): the 4000-atom LJ fluid, the 8000-ion Ewald
electrolyte (alpha 0.3, real-space cutoff 10, list radius 10.3, kmax 8:
4096 k-vectors, ~572 list entries per atom) and the 1,048,576-atom LJ
fluid.  Fixtures tests/golden/ref_bench_*.npz hold the unmodified
reference's output on exactly these states (tests/golden/make_golden.py):
the SHA-256 of its canonical pair set, its accelerations (every 64th atom of
the 1M system), virial, kinetic energy, S(k), k-space and self energies and
short trajectories under its own rebuild trigger (the LJ force states
displace the lattice sites by up to 0.1, since every force vanishes on the
perfect lattice; trajectories start from the benchmark states).  Energies the reference
does not compute (LJ of its force-shifted potential, Ewald real space over
the list) come from the FP64 C restatement at test time.

Tolerances:
  * pair sets: bit-exact (same digest and count);
  * FP64 form: accelerations 1e-12 (global relative), energies/virial 1e-11;
  * mixed form: ||dF|| / ||F|| <= 1e-5 and max_i |dF_i| <= 1e-5 rms|F|;
    energies/virial 1e-5 relative; S(k) 1e-5 of max |S|;
  * trajectories (positions; velocities 100x looser): 3 ion steps within
    1e-9 (FP64) / 1e-6 (mixed); 100 LJ steps within 1e-9 (FP64) / 1e-5
    (mixed; the fluid's chaotic growth over t = 0.5 amplifies the FP32
    rounding; measured 3e-7).
"""
import hashlib
import json

import numpy as np
import pytest

from helpers import force_errors, golden_path

pytestmark = pytest.mark.gpu

PRECS = ["mixed", "fp64"]


def digest(pairs):
    return hashlib.sha256(np.ascontiguousarray(pairs, dtype="<i4").tobytes()).hexdigest()


def fixture(name, run=False):
    """(system, fixture): the force state (generator with the fixture's
    keyword arguments) or, with run=True, the benchmark state itself."""
    from caviar_b200 import workloads as W
    d = np.load(golden_path(f"ref_bench_{name}.npz"))
    kw = {} if run else json.loads(str(d["generator_kwargs"]))
    s = getattr(W, str(d["generator"]))(**kw)
    assert s.n == int(d["n"])
    return s, d


def make(abi, s, prec, policy=None):
    p = abi.PREC_FP64 if prec == "fp64" else abi.PREC_MIXED
    pol = abi.REBUILD_DISPLACEMENT if policy is None else policy
    return abi.Simulation(s, precision=p, policy=pol)


def check_acc(acc, ref, prec):
    g, mx, _ = force_errors(acc, ref)
    print(f"force error {prec}: global {g:.3e}, max/rms {mx:.3e}")
    if prec == "fp64":
        assert g < 1e-12, (g, mx)
    else:
        assert g <= 1e-5 and mx <= 1e-5, (g, mx)


def rel(a, b):
    return abs(a - b) / abs(b)


def wrap_diff(a, b, L):
    d = a - b
    return d - L * np.round(d / L)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("name", ["lj4000", "ions8000", "lj1m"])
def test_bench_pair_set_forces_virial(cuda_lib, oracle_lib, name, prec):
    s, d = fixture(name)
    sim = make(cuda_lib, s, prec)
    acc, th = sim.compute_forces()
    pairs = sim.pairs()
    assert pairs.shape[0] == int(d["npairs"])
    assert digest(pairs) == str(d["pairs_sha256"])
    del pairs
    stride = int(d["acc_stride"])
    check_acc(acc[::stride], d["ref_acc"], prec)
    tol = 1e-11 if prec == "fp64" else 1e-5
    assert rel(th["virial"], float(d["ref_virial"])) <= tol, (th["virial"], float(d["ref_virial"]))
    assert rel(th["ke"], float(d["ref_ke"])) <= 1e-12
    o = oracle_lib.Oracle(s)
    o.setup()
    e = o.energy()
    scale = abs(e["e_lj"]) + abs(e["e_ewald_r"])
    assert abs(th["e_lj"] - e["e_lj"]) <= tol * scale, (th["e_lj"], e["e_lj"])
    assert abs(th["e_ewald_r"] - e["e_ewald_r"]) <= tol * scale, (th["e_ewald_r"], e["e_ewald_r"])
    if s.ewald_k is not None:
        sk = sim.sk()
        ref_sk = d["ref_sk"][0::2] + 1j * d["ref_sk"][1::2]
        assert len(sk) == len(ref_sk) == 4096
        assert np.abs(sk - ref_sk).max() <= (1e-11 if prec == "fp64" else 1e-5) * np.abs(ref_sk).max()
        assert rel(th["e_ewald_k"], float(d["ref_ek"])) <= tol
        assert rel(th["e_self"], float(d["ref_eself"])) <= 1e-12
    sim.close()


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("name", ["lj4000", "ions8000"])
def test_bench_trajectory_vs_reference(cuda_lib, name, prec):
    """The reference's own run (md_simulator step with its rebuild trigger)
    against cvr_run under CVR_REBUILD_REFERENCE."""
    s, d = fixture(name, run=True)
    nsteps = int(d["run_steps"])
    sim = make(cuda_lib, s, prec, policy=cuda_lib.REBUILD_REFERENCE)
    th = sim.run(nsteps, 1)
    pos, vel, _ = sim.state()
    dp = np.abs(wrap_diff(pos, d["run_pos"], s.box)).max()
    dv = np.abs(vel - d["run_vel"]).max()
    print(f"{name} {prec}: {nsteps} steps, max |dr| {dp:.3e}, max |dv| {dv:.3e}")
    if name == "lj4000":
        tol = 1e-9 if prec == "fp64" else 1e-5
    else:
        tol = 1e-9 if prec == "fp64" else 1e-6
    assert dp < tol and dv < 100 * tol
    # the kinetic-energy trace of every step
    ke = th[:, 1]
    ke_ref = np.asarray(d["run_ke"])[-nsteps:]
    assert np.abs(ke - ke_ref).max() <= (1e-9 if prec == "fp64" else 1e-4) * np.abs(ke_ref).max()
