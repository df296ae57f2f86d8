"""The CASL front end (cvr_casl_run_file): reference scripts for the hot-path
objects run on the GPU path unchanged.

CPU: scripts with off-path objects or unknown keywords are rejected with a
message (before any GPU work).  GPU: the script written with the reference's
own keywords (oracle.casl_script, the same text the reference harness runs)
plus atoms from an xyz file reproduces the reference's 20-step trajectory.
"""
import os

import numpy as np
import pytest

from helpers import load_ref_fixture


def write_xyz(path, s):
    with open(path, "w") as f:
        f.write(f"{s.n}\nstate\n")
        for t, p, v in zip(s.type, s.pos, s.vel):
            vals = " ".join(repr(float(x)) for x in (*p, *v))
            f.write(f"{int(t)} {vals}\n")


def script_for(s, tmp, nsteps, extra=()):
    from oracle import oracle as O
    body = O.casl_script(s, nsteps)
    body = body.replace("adata set_domain dom\n",
                        'adata set_domain dom\nadata add_xyz_data_file file_name "state.xyz" read_velocity\n')
    body += "\n".join(extra) + "\nsim run\nexit\n"
    write_xyz(os.path.join(tmp, "state.xyz"), s)
    path = os.path.join(tmp, "run.casl")
    with open(path, "w") as f:
        f.write(body)
    return path


def test_rejects_off_path_objects(cuda_lib, tmp_path):
    p = tmp_path / "bad.casl"
    p.write_text("domain box dom\nwriter atom_data w1\n")
    with pytest.raises(cuda_lib.CvrError) as e:
        cuda_lib.run_casl(str(p))
    assert "not on the B200 hot path" in str(e.value) and "bad.casl:2" in str(e.value)


def test_rejects_unknown_keyword(cuda_lib, tmp_path):
    p = tmp_path / "bad.casl"
    p.write_text("real rc 2.5\nneighborlist basic nl\nnl cutoff rc\nnl all_atom_test\n")
    with pytest.raises(cuda_lib.CvrError) as e:
        cuda_lib.run_casl(str(p))
    assert "all_atom_test" in str(e.value)


def test_requires_integrator_type(cuda_lib, tmp_path):
    s, _ = load_ref_fixture("lj500")
    from oracle import oracle as O
    body = O.casl_script(s, 5).replace("sim integrator_type velocity_verlet\n", "") + "sim run\n"
    (tmp_path / "state.xyz").write_text("1\nx\n0 1 1 1\n")
    p = tmp_path / "r.casl"
    p.write_text(body)
    with pytest.raises(cuda_lib.CvrError) as e:
        cuda_lib.run_casl(str(p))
    assert "integrator_type" in str(e.value)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["lj500", "ions500"])
def test_reference_script_reproduces_reference_trajectory(cuda_lib, tmp_path, name):
    s, d = load_ref_fixture(name)
    nsteps = int(d["run_steps"])
    path = script_for(s, str(tmp_path), nsteps, ["sim precision fp64", "sim rebuild_policy reference",
                                                  'sim state_file "out.bin"', "sim thermo_step 5",
                                                  'sim thermo_file "thermo.txt"'])
    cuda_lib.run_casl(path)
    raw = np.fromfile(tmp_path / "out.bin", dtype=np.float64, offset=8)
    n = s.n
    pos = raw[:3 * n].reshape(n, 3)
    L = s.box
    dp = pos - d["run_pos"].reshape(-1, 3)
    dp -= L * np.round(dp / L)
    assert np.abs(dp).max() < 1e-9
    th = np.loadtxt(tmp_path / "thermo.txt")
    assert th.shape == (nsteps // 5, 10)
    assert abs(th[-1, 1] - float(d["run_ke"][-1])) < 1e-8 * float(d["run_ke"][-1])
