"""GPU parity of the sm_100a path (through the C ABI) against the reference.

Oracles: the unmodified reference's own outputs (tests/golden/ref_*.npz,
produced by oracle/_ref built from the reference sources), the published
Ewald known answer (tests/golden/ewald_n100.json), and the FP64 C
restatement (oracle/) for cases without a fixture.

Tolerances (stated here, used below):
  * pair sets: bit-exact (same sorted canonical pair set);
  * FP64 form: accelerations within 1e-12 relative (global), energies/virial 1e-11;
  * mixed form: global relative force error ||dF|| / ||F|| <= 1e-5 and
    per-atom max |dF_i| <= 1e-5 * rms|F|; energies/virial 1e-5 relative.
"""
import numpy as np
import pytest

from helpers import ewald_golden, force_errors, load_ref_fixture

pytestmark = pytest.mark.gpu

FIXTURES = ["lj500", "ljmix500", "ions500"]
PRECS = ["mixed", "fp64"]


def sim_for(abi, s, prec, policy=None):
    p = abi.PREC_FP64 if prec == "fp64" else abi.PREC_MIXED
    pol = abi.REBUILD_DISPLACEMENT if policy is None else policy
    return abi.Simulation(s, precision=p, policy=pol)


def check_forces(acc, ref, prec):
    g, mx, _ = force_errors(acc, ref)
    if prec == "fp64":
        assert g < 1e-12, (g, mx)
    else:
        assert g <= 1e-5, (g, mx)
        assert mx <= 1e-5, (g, mx)
    return g, mx


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("name", FIXTURES)
def test_pair_set_bit_exact(cuda_lib, name, prec):
    s, d = load_ref_fixture(name)
    sim = sim_for(cuda_lib, s, prec)
    sim.build_neighbors(True)
    assert np.array_equal(sim.pairs(), d["ref_pairs"])


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("name", FIXTURES)
def test_forces_energy_virial_vs_reference(cuda_lib, oracle_lib, name, prec):
    s, d = load_ref_fixture(name)
    sim = sim_for(cuda_lib, s, prec)
    acc, th = sim.compute_forces()
    check_forces(acc, d["ref_acc"].reshape(-1, 3), prec)
    tol = 1e-11 if prec == "fp64" else 1e-5
    assert abs(th["virial"] - float(d["ref_virial"])) <= tol * abs(float(d["ref_virial"]))
    assert abs(th["ke"] - float(d["ref_ke"])) <= 1e-12 * abs(float(d["ref_ke"]))
    o = oracle_lib.Oracle(s)
    o.setup()
    e = o.energy()
    scale = abs(e["e_lj"]) + abs(e["e_ewald_r"]) + 1.0
    assert abs(th["e_lj"] - e["e_lj"]) <= tol * scale
    assert abs(th["e_ewald_r"] - e["e_ewald_r"]) <= tol * scale
    if s.ewald_k is not None:
        assert abs(th["e_ewald_k"] - float(d["ref_ek"])) <= tol * abs(float(d["ref_ek"]))
        assert abs(th["e_self"] - float(d["ref_eself"])) <= 1e-12 * abs(float(d["ref_eself"]))
        sk = sim.sk()
        ref_sk = d["ref_sk"][0::2] + 1j * d["ref_sk"][1::2]
        assert np.abs(sk - ref_sk).max() <= (1e-11 if prec == "fp64" else 1e-5) * np.abs(ref_sk).max()


@pytest.mark.parametrize("prec", PRECS)
def test_golden_ewald_known_answer(cuda_lib, prec):
    s, force, energy = ewald_golden()
    sim = sim_for(cuda_lib, s, prec)
    acc, th = sim.compute_forces()
    check_forces(acc, force, prec)
    e = th["e_ewald_r"] + th["e_ewald_k"] + th["e_self"]
    assert abs(e - energy) <= (1e-10 if prec == "fp64" else 1e-5) * abs(energy)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("name", FIXTURES)
def test_trajectory_vs_reference(cuda_lib, name, prec):
    """20 velocity-Verlet steps under the reference's rebuild policy."""
    s, d = load_ref_fixture(name)
    sim = sim_for(cuda_lib, s, prec, policy=cuda_lib.REBUILD_REFERENCE)
    sim.run(int(d["run_steps"]))
    pos, vel, acc = sim.state()
    L = s.box
    dp = pos - d["run_pos"].reshape(-1, 3)
    dp -= L * np.round(dp / L)
    tol_p = 1e-9 if prec == "fp64" else 1e-5
    assert np.abs(dp).max() < tol_p
    g, _, _ = force_errors(acc, d["run_acc"].reshape(-1, 3))
    assert g < (1e-8 if prec == "fp64" else 1e-4)


def test_reference_policy_rebuild_count(cuda_lib, oracle_lib):
    s, d = load_ref_fixture("lj500")
    o = oracle_lib.Oracle(s, policy=oracle_lib.POLICY_REFERENCE)
    o.setup()
    o.step(int(d["run_steps"]))
    sim = sim_for(cuda_lib, s, "fp64", policy=cuda_lib.REBUILD_REFERENCE)
    sim.run(int(d["run_steps"]))
    assert sim.info()["builds"] == int(o.scalars()["n_builds"])


@pytest.mark.parametrize("prec", PRECS)
def test_lj4000_vs_oracle(cuda_lib, oracle_lib, prec):
    from caviar_b200 import workloads as W
    s = W.fcc_lattice(10, 0.8442, 0.72, seed=1, jitter=0.1)
    o = oracle_lib.Oracle(s)
    o.setup()
    sim = sim_for(cuda_lib, s, prec)
    acc, th = sim.compute_forces()
    assert np.array_equal(sim.pairs(), o.pairs())
    check_forces(acc, o.state()[2], prec)


@pytest.mark.parametrize("stretch_z,bc", [(1.0, (1, 1, 1)), (1.07, (1, 1, 1)), (1.0, (1, 1, 0))])
def test_fixed_point_and_cell_local_forms(cuda_lib, oracle_lib, stretch_z, bc):
    """The mixed form takes fixed-point pair displacements in a cubic box
    (periodic or not: a listed pair never spans half the box, so the integer
    wrap never applies to it) and the cell-local FP32 form otherwise; both
    stay within the mixed tolerance of the FP64 oracle (forces, LJ energy,
    virial), and so does a 60-step run (positions within 1e-5, forces 1e-4,
    FP64 form the comparison)."""
    from caviar_b200 import workloads as W
    s = W.fcc_lattice(10, 0.8442, 0.72, seed=4, jitter=0.1)
    s.bc = bc
    s.hi = np.asarray(s.lo, np.float64) + s.box * np.array([1.0, 1.0, stretch_z])
    o = oracle_lib.Oracle(s)
    o.setup()
    sim = sim_for(cuda_lib, s, "mixed")
    acc, th = sim.compute_forces()
    assert sim.info()["fixed_point"] == (1 if stretch_z == 1.0 else 0)
    assert np.array_equal(sim.pairs(), o.pairs())
    check_forces(acc, o.state()[2], "mixed")
    sc = o.energy()
    assert abs(th["e_lj"] - sc["e_lj"]) <= 1e-5 * abs(sc["e_lj"])
    assert abs(th["virial"] - sc["virial"]) <= 1e-5 * abs(sc["virial"])
    ref = sim_for(cuda_lib, s, "fp64")
    assert ref.info()["fixed_point"] == 0
    sim.run(60)
    ref.run(60)
    p1, _, a1 = sim.state()
    p2, _, a2 = ref.state()
    dp = p1 - p2
    dp -= s.box * np.round(dp / s.box)
    assert np.abs(dp).max() < 1e-5
    assert force_errors(a1, a2)[0] < 1e-4


def test_fine_grid_box_uses_cell_local_form(cuda_lib, oracle_lib):
    """A cubic box with more than 256 cells per axis (a 4000-atom lattice
    cluster in L = 400: 285 cells) keeps the cell-local FP32 form, because
    the fixed-point step L / 2^32 would be coarser than the FP32 spacing of
    cell-local coordinates; pair set bit-exact, forces within the mixed
    tolerance of the FP64 oracle."""
    from caviar_b200 import workloads as W
    s = W.fcc_lattice(10, 0.8442, 0.72, seed=6, jitter=0.1)
    s.pos = s.pos + (200.0 - 0.5 * s.box[0])
    s.lo, s.hi = np.zeros(3), np.full(3, 400.0)
    o = oracle_lib.Oracle(s)
    o.setup()
    sim = sim_for(cuda_lib, s, "mixed")
    acc, _ = sim.compute_forces()
    info = sim.info()
    assert info["ncx"] > 256 and info["fixed_point"] == 0
    assert np.array_equal(sim.pairs(), o.pairs())
    check_forces(acc, o.state()[2], "mixed")


LIST_KERNELS = ["thread", "warp"]


def _lattice(nc, bc=(1, 1, 1), seed=5):
    from caviar_b200 import workloads as W
    s = W.fcc_lattice(nc, 0.8442, 0.72, seed=seed, jitter=0.1)
    s.bc = bc
    return s


@pytest.mark.parametrize("nc,bc", [(10, (1, 1, 1)), (10, (1, 0, 1)), (3, (1, 1, 1)), (3, (0, 1, 1))])
def test_list_kernels_same_pair_set(cuda_lib, oracle_lib, nc, bc):
    """Both list-search kernels (one thread per atom, one warp per atom)
    build the reference's pair set, and the FP64 forces from their lists
    agree to rounding (the 108-atom box has fewer than 2R + 1 cells per
    axis, so every stencil cell is searched as its own piece, with images)."""
    s = _lattice(nc, bc)
    o = oracle_lib.Oracle(s)
    o.setup()
    ref = o.pairs()
    acc = {}
    for name in LIST_KERNELS:
        kind = getattr(cuda_lib, "LIST_" + name.upper())
        sim = cuda_lib.Simulation(s, precision=cuda_lib.PREC_FP64, list_kernel=kind)
        a, _ = sim.compute_forces()
        assert np.array_equal(sim.pairs(), ref), name
        acc[name] = a
        sim.close()
    for name in LIST_KERNELS[1:]:
        assert force_errors(acc[name], acc["thread"])[0] < 1e-13


def test_list_kernels_atoms_outside_open_face(cuda_lib, oracle_lib):
    """Atoms beyond a non-periodic face are binned into the edge cells; the
    warp kernel's per-row clipping assumes every atom inside its cell, so a
    build that clamps one searches whole rows: both kernels keep the pair of
    two atoms outside the face, and the reference's pair set."""
    s = _lattice(10, (1, 0, 1))
    L = s.box
    s.pos[0] = [3.0, L[1] + 0.6, 4.0]
    s.pos[1] = [3.5, L[1] + 0.9, 4.2]
    s.pos[2] = [8.0, -0.4, 8.0]
    o = oracle_lib.Oracle(s)
    o.setup()
    ref = o.pairs()
    assert ((ref[:, 0] == 0) & (ref[:, 1] == 1)).any() or ((ref[:, 0] == 1) & (ref[:, 1] == 0)).any()
    for name in LIST_KERNELS:
        sim = cuda_lib.Simulation(s, precision=cuda_lib.PREC_FP64, list_kernel=getattr(cuda_lib, "LIST_" + name.upper()))
        sim.build_neighbors(True)
        assert np.array_equal(sim.pairs(), ref), name
        sim.close()


def test_list_kernels_large_system_and_run(cuda_lib):
    """186,624 atoms (the size class where one thread per atom is the
    default): the warp kernel gives the same pair set at setup, and after a
    50-step run with several rebuilds the trajectories agree to FP32
    rounding and the lists to pairs within rounding of rl."""
    s = _lattice(36)
    out = {}
    for name in ("thread", "warp"):
        kind = getattr(cuda_lib, "LIST_" + name.upper())
        sim = cuda_lib.Simulation(s, precision=cuda_lib.PREC_MIXED, list_kernel=kind)
        sim.build_neighbors(True)
        p0 = sim.pairs()
        sim.run(50)
        assert sim.info()["builds"] >= 3
        sim.build_neighbors(True)
        out[name] = (p0, sim.pairs(), sim.state())
        sim.close()
    assert np.array_equal(out["thread"][0], out["warp"][0])
    pa, pb = out["thread"][2][0], out["warp"][2][0]
    dp = pa - pb
    dp -= s.box * np.round(dp / s.box)
    assert np.abs(dp).max() < 1e-5
    # after identical-to-rounding runs the two lists may differ only by pairs within rounding of rl
    a, b = out["thread"][1], out["warp"][1]
    assert abs(len(a) - len(b)) <= 1e-5 * len(a)


@pytest.mark.parametrize("name", ["lj500", "ions500"])
def test_set_state_again_matches_fresh_context(cuda_lib, name):
    """A context whose state is set again (same atom count and settings:
    cells, tables and step graphs are kept) continues exactly like a fresh
    context given that state: trajectories and thermo (self energy
    included) bit-identical."""
    s, _ = load_ref_fixture(name)
    a = sim_for(cuda_lib, s, "mixed")
    a.run(25, 25)
    a.set_state(s.pos, s.vel, s.type, s.mol)
    ta = a.run(25, 25)
    b = sim_for(cuda_lib, s, "mixed")
    tb = b.run(25, 25)
    for x, y in zip(a.state(), b.state()):
        assert np.array_equal(x, y)
    assert np.array_equal(ta, tb)
    if s.ewald_k is not None:
        assert ta[0, cuda_lib.TH_KEYS.index("e_self")] != 0.0


def test_deterministic(cuda_lib):
    from caviar_b200 import workloads as W
    s = W.config_lj_4000()
    out = []
    for _ in range(2):
        sim = sim_for(cuda_lib, s, "mixed")
        sim.run(50)
        out.append(sim.state())
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_edge_cases(cuda_lib):
    from caviar_b200 import workloads as W
    s = W.fcc_lattice(3, 0.8442, 0.5, seed=1)
    one = s.copy()
    one.pos, one.vel, one.type = s.pos[:1], s.vel[:1], s.type[:1]
    sim = sim_for(cuda_lib, one, "mixed")
    acc, _ = sim.compute_forces()
    assert sim.pairs().shape == (0, 5) and np.all(acc == 0)
    L = float(s.box[0])
    two = s.copy()
    two.pos = np.array([[0.5, 1.0, 1.0], [L - 0.5, 1.0, 1.0]])
    two.vel = np.zeros((2, 3))
    two.type = np.zeros(2, np.int32)
    sim = sim_for(cuda_lib, two, "fp64")
    acc, _ = sim.compute_forces()
    assert sim.pairs().tolist() == [[0, 1, -1, 0, 0]]
    assert acc[0, 0] > 0 and acc[1, 0] < 0
    face = two.copy()
    face.pos = np.array([[L, 1.0, 1.0], [L - 1.0, 1.0, 1.0]])
    sim = sim_for(cuda_lib, face, "fp64")
    sim.build_neighbors(True)
    assert sim.pairs().shape[0] == 1


def test_nan_is_reported(cuda_lib):
    from caviar_b200 import workloads as W
    s = W.fcc_lattice(3, 0.8442, 0.5, seed=1)
    s.pos = s.pos.copy()
    s.pos[1] = s.pos[0]  # coincident LJ atoms -> infinite / NaN force
    sim = sim_for(cuda_lib, s, "mixed")
    with pytest.raises(cuda_lib.CvrError) as e:
        sim.run(2)
    assert e.value.code == 3


def test_list_overflow_regrows(cuda_lib, oracle_lib):
    """Compress the atoms after the first build so the next build needs a
    longer list than the first one sized: the list regrows and the pair set
    still matches the oracle."""
    from caviar_b200 import workloads as W
    s = W.fcc_lattice(4, 0.3, 0.0, seed=1)
    sim = sim_for(cuda_lib, s, "fp64")
    sim.build_neighbors(True)
    cap0 = sim.info()["cap"]
    pos = s.lo + (s.pos - s.lo) * 0.6
    sim.set_state(pos, np.zeros_like(pos), s.type)
    sim.build_neighbors(True)
    assert sim.info()["cap"] > cap0
    s2 = s.copy()
    s2.pos = pos
    o = oracle_lib.Oracle(s2)
    o.build_list()
    assert np.array_equal(sim.pairs(), o.pairs())


def test_graph_and_stream_paths_agree(cuda_lib):
    """cvr_run replays one CUDA graph per step (list build in a conditional
    node); with kernel timing on it launches the same kernels on the stream.
    Both must give the same trajectory and thermo records, bit for bit."""
    from caviar_b200 import workloads as W
    s = W.fcc_lattice(8, 0.8442, 0.72, seed=5, jitter=0.05)
    a = sim_for(cuda_lib, s, "mixed")
    th_a = a.run(60, 10)
    b = sim_for(cuda_lib, s, "mixed")
    b.set_kernel_timing(True)
    th_b = b.run(60, 10)
    for x, y in zip(a.state(), b.state()):
        assert np.array_equal(x, y)
    assert np.array_equal(th_a, th_b)
    assert a.info()["builds"] == b.info()["builds"] > 1
    # thermo records: step numbers, and the last KE equals the state's
    assert th_a[:, 0].tolist() == [10, 20, 30, 40, 50, 60]
    _, vel, _ = a.state()
    v = vel - vel.mean(axis=0)
    assert abs(th_a[-1, 1] - 0.5 * np.sum(v * v)) < 1e-10 * th_a[-1, 1]


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_deferred_kick_matches_separate_kicks(cuda_lib, prec):
    """Inside one cvr_run a plain step (no thermo record, not the last) leaves
    its second half kick to the next step's kick-drift kernel, which applies
    it first with the same acceleration.  The trajectory must equal, bit for
    bit, runs of one step each (whose step always ends with its own kick)."""
    from caviar_b200 import workloads as W
    s = W.fcc_lattice(8, 0.8442, 0.72, seed=11, jitter=0.05)
    a = sim_for(cuda_lib, s, prec)
    a.run(40)
    b = sim_for(cuda_lib, s, prec)
    for _ in range(40):
        b.run(1)
    for x, y in zip(a.state(), b.state()):
        assert np.array_equal(x, y)
    assert a.info()["builds"] == b.info()["builds"] > 1
    # a run that ends on a thermo record, then one that does not: same state
    c = sim_for(cuda_lib, s, prec)
    th = c.run(30, 15)
    c.run(10)
    for x, y in zip(a.state(), c.state()):
        assert np.array_equal(x, y)
    assert th[:, 0].tolist() == [15, 30]


def test_changed_dt_reaches_the_step_graphs(cuda_lib):
    """cvr_set_integrator between two runs: the graph path (which bakes dt
    and k_b into its kernels) must follow the new values exactly like the
    stream path, which reads them at every launch."""
    from caviar_b200 import workloads as W
    s = W.fcc_lattice(6, 0.8442, 0.72, seed=9, jitter=0.05)
    a = sim_for(cuda_lib, s, "mixed")
    b = sim_for(cuda_lib, s, "mixed")
    b.set_kernel_timing(True)
    for sim in (a, b):
        sim.run(20)
        sim.set_integrator(0.5 * s.dt, 2.0)
    th_a = a.run(20, 10)
    th_b = b.run(20, 10)
    for x, y in zip(a.state(), b.state()):
        assert np.array_equal(x, y)
    assert np.array_equal(th_a, th_b)
    # and the run really used the new values: a fresh context with them from the start
    c = sim_for(cuda_lib, s, "mixed")
    c.set_integrator(s.dt, 2.0)
    c.run(20)
    c.set_integrator(0.5 * s.dt, 2.0)
    th_c = c.run(20, 10)
    assert np.array_equal(th_a, th_c)


@pytest.mark.parametrize("prec", PRECS)
def test_lj_jump_tol_vs_reference(cuda_lib, prec):
    """cvr_set_lj_jump_tol (lj.cpp:118-127, 423-432) against the unmodified
    reference's forces and virial on a fluid with pairs closer than
    sqrt(jump_tol) (tests/golden/ref_ljjump500.npz); the clamp takes the
    multi-type pair kernel."""
    import importlib.util
    import os
    from helpers import GOLDEN
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    d = np.load(os.path.join(GOLDEN, "ref_ljjump500.npz"))
    s = mg.jump_system()
    assert np.array_equal(s.pos, d["pos"])
    sim = sim_for(cuda_lib, s, prec)
    acc, th = sim.compute_forces()
    check_forces(acc, d["acc"], prec)
    tol = 1e-11 if prec == "fp64" else 1e-5
    assert abs(th["virial"] - float(d["virial"])) <= tol * abs(float(d["virial"]))


@pytest.mark.parametrize("prec", PRECS)
def test_all_atom_test_vs_reference(cuda_lib, prec):
    """cvr_set_all_atom_test (neighborlist.cpp:161-191): the pair set of every
    owned pair and ghost image, forces, virial, S(k) and a 10-step run under
    the reference's rebuild trigger against the unmodified reference with
    `neigh all_atom_test` (tests/golden/ref_allatom300.npz)."""
    import hashlib
    import importlib.util
    import os
    from helpers import GOLDEN
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    d = np.load(os.path.join(GOLDEN, "ref_allatom300.npz"))
    s = mg.all_atom_system()
    sim = sim_for(cuda_lib, s, prec, policy=cuda_lib.REBUILD_REFERENCE)
    sim.set_all_atom_test(True)
    acc, th = sim.compute_forces()
    p = sim.pairs()
    assert p.shape[0] == int(d["npairs"])
    assert hashlib.sha256(np.ascontiguousarray(p, dtype="<i4").tobytes()).hexdigest() == str(d["pairs_sha256"])
    check_forces(acc, d["acc"], prec)
    tol = 1e-11 if prec == "fp64" else 1e-5
    assert abs(th["virial"] - float(d["virial"])) <= tol * abs(float(d["virial"]))
    sk = sim.sk()
    ref_sk = d["sk"][0::2] + 1j * d["sk"][1::2]
    assert np.abs(sk - ref_sk).max() <= (1e-11 if prec == "fp64" else 1e-5) * np.abs(ref_sk).max()
    sim.run(int(d["run_steps"]))
    pos, _, _ = sim.state()
    dp = pos - d["run_pos"]
    dp -= s.box * np.round(dp / s.box)
    assert np.abs(dp).max() < (1e-9 if prec == "fp64" else 1e-5), np.abs(dp).max()


def test_type_out_of_range_rejected_and_state_kept(cuda_lib):
    """cvr_set_state checks every type on the GPU (atoms per type) before the
    staged arrays reach the state: a type outside [0, n_types) is
    CVR_ERR_INVALID and the context keeps its previous state (a run
    continues from it)."""
    s, _ = load_ref_fixture("lj500")
    sim = sim_for(cuda_lib, s, "fp64")
    p0, v0, _ = sim.state()
    bad = np.array(s.type, np.int32).copy()
    bad[123] = s.n_types + 2
    with pytest.raises(cuda_lib.CvrError) as e:
        sim.set_state(s.pos + 0.01, s.vel, bad)
    assert "type out of range" in str(e.value)
    p1, v1, _ = sim.state()
    assert np.array_equal(p0, p1) and np.array_equal(v0, v1)
    ref = sim_for(cuda_lib, s, "fp64")
    sim.run(5)
    ref.run(5)
    assert np.array_equal(sim.state()[0], ref.state()[0])
