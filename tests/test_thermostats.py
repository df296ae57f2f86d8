"""Thermostat constraints on the velocity-Verlet step: the reference's
`constraint berendsen` and `constraint nose_hoover` (constraint/berendsen.cpp,
constraint/nose_hoover.cpp), applied where Md_simulator calls
apply_thermostat (md_simulator.cpp:619-627).

GPU: 30-step trajectories (positions, velocities, kinetic-energy trace, and
the thermostat-modified accelerations for Nose-Hoover) match the unmodified
reference's (tests/golden/ref_{berendsen,nosehoover}500.npz), through the C
ABI and through CASL scripts; long runs hold the target temperature.
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


def attach(sim, name):
    if name == "berendsen500":
        sim.set_berendsen(1.2, 0.1, 0.005, step=2)
    else:
        sim.set_nose_hoover(1.2, 0.005, type=1, mass=20.0, kb=1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["berendsen500", "nosehoover500"])
@pytest.mark.parametrize("prec,tol", [(1, 1e-9), (0, 1e-6)])
def test_matches_reference(cuda_lib, name, prec, tol):
    d = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    s = fluid()
    sim = cuda_lib.Simulation(s, precision=prec, policy=cuda_lib.REBUILD_REFERENCE)
    attach(sim, name)
    th = sim.run(int(d["nsteps"]), thermo_every=1)
    pos, vel, acc = sim.state()
    assert np.abs(wrapped_diff(pos, d["pos"], s.box)).max() < tol
    assert np.abs(vel - d["vel"]).max() < 10 * tol
    assert np.allclose(th[:, cuda_lib.TH_KEYS.index("ke")], d["ke"], rtol=10 * tol, atol=0)
    if name == "nosehoover500":
        assert np.abs(acc - d["acc"]).max() < 100 * tol * np.abs(d["acc"]).max()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["berendsen500", "nosehoover500"])
def test_casl_thermostat_script(cuda_lib, tmp_path, name):
    from oracle import oracle as O
    from test_casl import write_xyz
    d = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    s = fluid()
    body = O.casl_script(s, int(d["nsteps"]), extra=str(d["script"]))
    body = body.replace("adata set_domain dom\n",
                        'adata set_domain dom\nadata add_xyz_data_file file_name "state.xyz" read_velocity\n')
    body += 'sim precision fp64\nsim rebuild_policy reference\nsim state_file "out.bin"\nsim run\nexit\n'
    write_xyz(str(tmp_path / "state.xyz"), s)
    (tmp_path / "run.casl").write_text(body)
    cuda_lib.run_casl(str(tmp_path / "run.casl"))
    raw = np.fromfile(tmp_path / "out.bin", dtype=np.float64, offset=8)
    assert np.abs(wrapped_diff(raw[:3 * s.n].reshape(-1, 3), d["pos"], s.box)).max() < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["berendsen", "nose_hoover"])
def test_holds_target_temperature(cuda_lib, kind):
    s = fluid()
    sim = cuda_lib.Simulation(s, precision=0)
    if kind == "berendsen":
        sim.set_berendsen(1.5, 0.1, 0.005)
    else:
        # type 1: zeta_dot = (kb n_df / Q)(T - T0), so <T> = T0; Q = n_df T0 tau^2 with tau = 0.5
        # (type 2's zeta_dot ~ (T0/T - 1) pins the harmonic mean of T instead)
        sim.set_nose_hoover(1.5, 0.005, type=1, mass=1497 * 1.5 * 0.25, kb=1.0)
    sim.run(3000)
    th = sim.run(12000, thermo_every=50)
    T = th[:, cuda_lib.TH_KEYS.index("temperature")]
    assert abs(T.mean() - 1.5) < 0.05 * 1.5, T.mean()
