"""Langevin velocity Verlet (the reference's integrator_type
velocity_verlet_langevin, md_simulator.cpp:670-811).

GPU: with the reference's own noise streams (std::mt19937 seeded 1, 2, 3,
std::normal_distribution, made on the host) a 20-step trajectory matches the
unmodified reference's (tests/golden/ref_langevin500.npz), through the C ABI
and through a CASL script; with the counter-based GPU generator the
thermostat holds the set temperature, and runs are reproducible per seed.
"""
import os

import numpy as np
import pytest

from caviar_b200 import workloads as W
from helpers import GOLDEN


def fluid():
    return W.fcc_lattice(5, 0.8442, 0.72, seed=7, jitter=0.05)


def wrapped_diff(a, b, L):
    d = a - b
    return d - L * np.round(d / L)


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [(1, 1e-9), (0, 1e-6)])
def test_reference_stream_matches_reference(cuda_lib, prec, tol):
    d = np.load(os.path.join(GOLDEN, "ref_langevin500.npz"))
    s = fluid()
    sim = cuda_lib.Simulation(s, precision=prec, policy=cuda_lib.REBUILD_REFERENCE)
    sim.set_langevin(1.2, 0.5, kb=1.0, rng=cuda_lib.RNG_REFERENCE)
    th = sim.run(int(d["nsteps"]), thermo_every=1)
    pos, vel, _ = sim.state()
    assert np.abs(wrapped_diff(pos, d["pos"], s.box)).max() < tol
    assert np.abs(vel - d["vel"]).max() < 10 * tol
    ke = th[:, cuda_lib.TH_KEYS.index("ke")]
    assert np.allclose(ke, d["ke"], rtol=10 * tol, atol=0)


@pytest.mark.gpu
def test_casl_langevin_script(cuda_lib, tmp_path):
    from oracle import oracle as O
    from test_casl import write_xyz
    d = np.load(os.path.join(GOLDEN, "ref_langevin500.npz"))
    s = fluid()
    body = O.casl_script(s, int(d["nsteps"]), extra=str(d["script"]))
    body = body.replace("adata set_domain dom\n",
                        'adata set_domain dom\nadata add_xyz_data_file file_name "state.xyz" read_velocity\n')
    body += 'sim precision fp64\nsim rebuild_policy reference\nsim state_file "out.bin"\nsim run\nexit\n'
    write_xyz(str(tmp_path / "state.xyz"), s)
    (tmp_path / "run.casl").write_text(body)
    cuda_lib.run_casl(str(tmp_path / "run.casl"))
    raw = np.fromfile(tmp_path / "out.bin", dtype=np.float64, offset=8)
    pos = raw[:3 * s.n].reshape(-1, 3)
    assert np.abs(wrapped_diff(pos, d["pos"], s.box)).max() < 1e-9


@pytest.mark.gpu
def test_philox_thermostat_holds_temperature(cuda_lib):
    s = fluid()
    sim = cuda_lib.Simulation(s, precision=0)
    sim.set_langevin(1.5, 1.0, kb=1.0, rng=cuda_lib.RNG_PHILOX, seed=12345)
    sim.run(2000)  # equilibrate (1/friction = 200 steps)
    th = sim.run(6000, thermo_every=50)
    T = th[:, cuda_lib.TH_KEYS.index("temperature")]
    assert abs(T.mean() - 1.5) < 0.06, T.mean()
    assert 0.01 < T.std() / T.mean() < 0.1


@pytest.mark.gpu
def test_philox_reproducible_per_seed(cuda_lib):
    s = fluid()
    out = []
    for seed in (7, 7, 8):
        sim = cuda_lib.Simulation(s, precision=0)
        sim.set_langevin(1.0, 0.5, kb=1.0, rng=cuda_lib.RNG_PHILOX, seed=seed)
        sim.run(50)
        out.append(sim.state()[1])
    assert np.array_equal(out[0], out[1])
    assert not np.array_equal(out[0], out[2])


@pytest.mark.gpu
def test_rejects_missing_temperature(cuda_lib):
    s = fluid()
    with pytest.raises(cuda_lib.CvrError):
        sim = cuda_lib.Simulation(s, precision=0)
        sim.set_langevin(-1.0, 0.5)
