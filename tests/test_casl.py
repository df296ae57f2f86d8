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

from caviar_b200 import workloads as W
from helpers import GOLDEN, load_ref_fixture


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
    p.write_text("domain box dom\nconstraint shake c1\n")
    with pytest.raises(cuda_lib.CvrError) as e:
        cuda_lib.run_casl(str(p))
    assert "not on the B200 hot path" in str(e.value) and "bad.casl:2" in str(e.value)


def test_rejects_unknown_keyword(cuda_lib, tmp_path):
    p = tmp_path / "bad.casl"
    p.write_text("real rc 2.5\nneighborlist basic nl\nnl cutoff rc\nnl bin_resize\n")
    with pytest.raises(cuda_lib.CvrError) as e:
        cuda_lib.run_casl(str(p))
    assert "bin_resize" in str(e.value)


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


def test_time_and_step_settings_are_exclusive(cuda_lib, tmp_path):
    """md_simulator takes its run length from steps or from times, not both
    (Md_simulator::verify_settings, md_simulator.cpp:276-282); atom_data
    msd_process is accepted."""
    s, _ = load_ref_fixture("lj500")
    from oracle import oracle as O
    body = O.casl_script(s, 5).replace("adata set_domain dom\n", "adata set_domain dom\nadata msd_process 1\n")
    body += "sim final_time 1.0\nsim run\n"
    p = tmp_path / "r.casl"
    p.write_text(body)
    with pytest.raises(cuda_lib.CvrError) as e:
        cuda_lib.run_casl(str(p))
    assert "cannot use both 'time' and 'step'" in str(e.value)


def test_final_step_add_alone_selects_no_run_length(cuda_lib, tmp_path):
    """final_step_add adds to final_step and restarts from the current step
    but, as in the reference (md_simulator.cpp:91-97), does not select step
    mode: a script with only final_step_add fails verify_settings."""
    s, _ = load_ref_fixture("lj500")
    from oracle import oracle as O
    body = O.casl_script(s, 5).replace("sim initial_step 0\n", "").replace("sim final_step 5\n", "")
    assert "final_step" not in body and "initial_step" not in body
    body += "sim final_step_add 5\nsim run\n"
    p = tmp_path / "r.casl"
    p.write_text(body)
    with pytest.raises(cuda_lib.CvrError) as e:
        cuda_lib.run_casl(str(p))
    assert "please assign 'time' or 'step' variables" in str(e.value)


@pytest.mark.gpu
def test_final_step_add_with_final_time(cuda_lib, tmp_path):
    """final_step_add restarts from the current step: `final_step 200, run,
    final_step_add 200, run` runs steps [0, 200) then [200, 400).  With
    final_time set, final_step_add is accepted and has no effect: each run
    recomputes its steps from the times ((int)1.0 / 0.005 = 200), as the
    reference's verify_settings does.  Both scripts end in the same state."""
    s, _ = load_ref_fixture("lj500")
    states = []
    for tag in ("step", "time"):
        d = tmp_path / tag
        d.mkdir()
        path = script_for(s, str(d), 200, [])
        text = open(path).read()
        if tag == "step":
            text = text.replace("sim run\n", 'sim run\nsim final_step_add 200\nsim state_file "out.bin"\nsim run\n', 1)
        else:
            text = text.replace("sim initial_step 0\n", "").replace("sim final_step 200\n", "")
            text = text.replace("sim run\n", "sim final_time 1.0\nsim final_step_add 3\nsim run\n"
                                'sim final_step_add 60\nsim state_file "out.bin"\nsim run\n', 1)
        open(path, "w").write(text)
        cuda_lib.run_casl(path)
        states.append(np.fromfile(d / "out.bin", dtype=np.float64, offset=8))
    assert np.array_equal(states[0], states[1])


@pytest.mark.gpu
def test_final_time_counts_steps_like_the_reference(cuda_lib, tmp_path):
    """final_time T runs (int)T / dt steps, the reference's conversion
    (md_simulator.cpp:508-512: the time is truncated before the division):
    final_time 1.9 at dt 0.005 ends in the state of final_step 200."""
    s, _ = load_ref_fixture("lj500")
    states = []
    for tag, extra in (("t", ["sim final_time 1.9"]), ("s", [])):
        d = tmp_path / tag
        d.mkdir()
        path = script_for(s, str(d), 200, extra + ['sim state_file "out.bin"'])
        if tag == "t":
            text = open(path).read().replace("sim initial_step 0\n", "").replace("sim final_step 200\n", "")
            assert "initial_step" not in text and "final_step" not in text
            open(path, "w").write(text)
        cuda_lib.run_casl(path)
        states.append(np.fromfile(d / "out.bin", dtype=np.float64, offset=8))
    assert np.array_equal(states[0], states[1])


def test_remove_objects_from_the_simulator(cuda_lib, tmp_path):
    """md_simulator remove_* drops the named object from the simulator's list
    (md_simulator.cpp:107-150): removing the only neighbour list leaves a
    simulator the B200 path refuses; removing an object the simulator does
    not hold is the reference's 'Unknown ... to remove.' error."""
    s, _ = load_ref_fixture("lj500")
    from oracle import oracle as O
    base = O.casl_script(s, 5)
    (tmp_path / "a.casl").write_text(base + "sim remove_neighborlist neigh\nsim run\n")
    with pytest.raises(cuda_lib.CvrError) as e:
        cuda_lib.run_casl(str(tmp_path / "a.casl"))
    assert "exactly one neighborlist" in str(e.value)
    (tmp_path / "b.casl").write_text(base + "sim remove_force_field f_lj\nsim remove_force_field f_lj\n")
    with pytest.raises(cuda_lib.CvrError) as e:
        cuda_lib.run_casl(str(tmp_path / "b.casl"))
    assert "Unknown force_field to remove." in str(e.value)


def test_add_random_velocity_matches_reference(cuda_lib, tmp_path):
    """atom_data add_random_velocity seed amplitude gives the velocities of
    the reference's own Atom_data::add_random_velocity (fixture from the
    unmodified reference: two species, masses 1 and 2.5, mass-weighted
    centre-of-mass removal) bit for bit; write_state_file dumps the prepared
    atoms (CPU: the script has no md_simulator run)."""
    d = np.load(os.path.join(GOLDEN, "ref_randvel500.npz"))
    L = float(d["box"][0])
    pos, typ = d["pos"], d["type"]
    with open(tmp_path / "state.xyz", "w") as f:
        f.write(f"{len(pos)}\nstate\n")
        for t, p in zip(typ, pos):
            f.write(f"{int(t)} " + " ".join(repr(float(x)) for x in p) + "\n")
    script = "\n".join([
        "domain box dom", f"dom xmin 0.0 xmax {L!r}", f"dom ymin 0.0 ymax {L!r}", f"dom zmin 0.0 zmax {L!r}",
        "dom boundary_condition 1 1 1", "dom generate", "atom_data basic adata", "adata set_domain dom",
        "adata add_type_mass 0 1.0", "adata add_type_mass 1 2.5",
        'adata add_xyz_data_file file_name "state.xyz"',
        f"adata add_random_velocity {int(d['seed'])} {float(d['amplitude'])!r}",
        'adata write_state_file "prepared.bin"', "exit", ""])
    (tmp_path / "rv.casl").write_text(script)
    cuda_lib.run_casl(str(tmp_path / "rv.casl"))
    raw = np.fromfile(tmp_path / "prepared.bin", dtype=np.float64, offset=8)
    n = len(pos)
    assert np.array_equal(raw[:3 * n].reshape(n, 3), pos)
    assert np.array_equal(raw[3 * n:6 * n].reshape(n, 3), d["vel"])


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


def test_rejects_unsupported_writer_keyword(cuda_lib, tmp_path):
    p = tmp_path / "bad.casl"
    p.write_text("writer atom_data w\nw msd_step 10\n")
    with pytest.raises(cuda_lib.CvrError) as e:
        cuda_lib.run_casl(str(p))
    assert "msd_step" in str(e.value)


def lj500_script(tmp, nsteps, extra, tail):
    from oracle import oracle as O
    s = W.fcc_lattice(5, 0.8442, 0.72, seed=7, jitter=0.05)
    body = O.casl_script(s, nsteps, extra=extra)
    body = body.replace("adata set_domain dom\n",
                        'adata set_domain dom\nadata add_xyz_data_file file_name "state.xyz" read_velocity\n')
    write_xyz(os.path.join(tmp, "state.xyz"), s)
    return body + tail


def parse_rows(text):
    return [line.split() for line in text.strip().splitlines()]


@pytest.mark.gpu
def test_writer_outputs_match_reference(cuda_lib, tmp_path):
    """writer atom_data: the energy, temperature, pressure, volume and xyz
    files of a 40-step run match the unmodified reference's own files
    (tests/golden/writer_lj500, 6 significant digits: compared to 1.1e-5)."""
    g = os.path.join(GOLDEN, "writer_lj500")
    extra = open(os.path.join(g, "script_extra.casl")).read()
    body = lj500_script(str(tmp_path), 40, extra, "sim precision fp64\nsim rebuild_policy reference\nsim run\nexit\n")
    (tmp_path / "run.casl").write_text(body)
    cuda_lib.run_casl(str(tmp_path / "run.casl"))
    for name in ("o_energy.txt", "o_temperature.txt", "o_pressure.txt", "o_volume.txt", "o_xyz.xyz"):
        ref = parse_rows(open(os.path.join(g, name)).read())
        got = parse_rows((tmp_path / name).read_text())
        assert len(got) == len(ref), name
        for a, b in zip(got, ref):
            assert len(a) == len(b), (name, a, b)
            if len(b) == 1:  # xyz header lines
                assert a == b
                continue
            x, y = np.array(a, float), np.array(b, float)
            assert np.allclose(x, y, rtol=1.1e-5, atol=1e-9), (name, a, b)


@pytest.mark.gpu
def test_restart_round_trips_bit_exactly(cuda_lib, tmp_path):
    """Checkpoints: an xyz frame written at 17 significant digits, read back
    with add_xyz_data_file last_frame replace_data, and the FP64 binary
    state_file read back with add_state_file replace_data, reproduce the
    final positions and velocities bit for bit."""
    t = str(tmp_path)
    w = ("writer atom_data w\nw set_atom_data adata\nw xyz_step 20\nw xyz_output_velocity 1\nw precision 17\n"
         "sim add_writer w\n")
    body = lj500_script(t, 21, w, 'sim rebuild_policy reference\nsim state_file "a.bin"\nsim run\nexit\n')
    (tmp_path / "a.casl").write_text(body)
    cuda_lib.run_casl(str(tmp_path / "a.casl"))
    # reload from the last xyz frame, run no step, dump
    body = lj500_script(t, 1, 'adata add_xyz_data_file file_name "o_xyz.xyz" last_frame replace_data read_velocity\n',
                        'sim final_step 0\nsim state_file "b.bin"\nsim run\nexit\n')
    (tmp_path / "b.casl").write_text(body)
    cuda_lib.run_casl(str(tmp_path / "b.casl"))
    body = lj500_script(t, 1, 'adata add_state_file file_name "a.bin" replace_data\n',
                        'sim final_step 0\nsim state_file "c.bin"\nsim run\nexit\n')
    (tmp_path / "c.casl").write_text(body)
    cuda_lib.run_casl(str(tmp_path / "c.casl"))
    a, b, c = (np.fromfile(tmp_path / f, dtype=np.float64) for f in ("a.bin", "b.bin", "c.bin"))
    n = 500
    assert int(a[:1].view(np.int64)[0]) == n
    pv = slice(1, 1 + 6 * n)  # positions and velocities
    assert np.array_equal(a[pv], b[pv])
    assert np.array_equal(a[pv], c[pv])
