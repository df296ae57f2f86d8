"""CPU: the FP64 restatement (oracle/) against the reference's golden data.

* the published Ewald known-answer case (benchmark/b2-ewald), and
* fixtures produced by the unmodified reference built from its own sources
  (tests/golden/ref_*.npz, generated by tests/golden/make_golden.py):
  bit-exact accelerations, pair sets, virial, kinetic energy, S(k), k-space
  and self energies, and a 20-step trajectory under the reference's rebuild
  policy.
"""
import os

import numpy as np
import pytest

from helpers import GOLDEN as GOLDEN_DIR
from helpers import ewald_golden, load_ref_fixture

FIXTURES = ["lj500", "ljmix500", "ions500"]


def test_golden_ewald_forces_and_energy(oracle_lib):
    O = oracle_lib
    s, force, energy = ewald_golden()
    o = O.Oracle(s)
    o.setup()
    _, _, acc = o.state()
    rel = np.linalg.norm(acc - force, axis=1) / np.linalg.norm(force, axis=1)
    assert rel.max() < 1e-10
    e = o.energy()
    assert abs(e["e_ewald_r"] + e["e_ewald_k"] + e["e_self"] - energy) < 1e-9 * abs(energy)


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_bit_exact_vs_reference_forces(oracle_lib, name):
    O = oracle_lib
    s, d = load_ref_fixture(name)
    o = O.Oracle(s)
    o.setup()
    _, _, acc = o.state()
    assert np.array_equal(acc, d["ref_acc"].reshape(-1, 3))
    assert np.array_equal(o.pairs(), d["ref_pairs"])
    sc = o.scalars()
    assert sc["virial"] == float(d["ref_virial"])
    assert sc["ke"] == float(d["ref_ke"])
    if s.ewald_k is not None:
        sk = d["ref_sk"]
        assert np.array_equal(o.sk(), sk[0::2] + 1j * sk[1::2])
        e = o.energy()
        assert e["e_ewald_k"] == float(d["ref_ek"])
        assert e["e_self"] == float(d["ref_eself"])


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_bit_exact_vs_reference_trajectory(oracle_lib, name):
    O = oracle_lib
    s, d = load_ref_fixture(name)
    o = O.Oracle(s, policy=O.POLICY_REFERENCE)
    o.setup()
    o.step(int(d["run_steps"]))
    pos, vel, acc = o.state()
    assert np.array_equal(pos, d["run_pos"].reshape(-1, 3))
    assert np.array_equal(vel, d["run_vel"].reshape(-1, 3))
    assert np.array_equal(acc, d["run_acc"].reshape(-1, 3))


def test_displacement_policy_same_trajectory(oracle_lib):
    """Rebuilding only on displacement (fewer builds) keeps the LJ trajectory
    (LJ has its own cutoff test, so the list content beyond rc is irrelevant)."""
    O = oracle_lib
    s, d = load_ref_fixture("lj500")
    o = O.Oracle(s, policy=O.POLICY_DISPLACEMENT)
    o.setup()
    o.step(int(d["run_steps"]))
    pos, vel, _ = o.state()
    L = s.box
    dp = pos - d["run_pos"].reshape(-1, 3)
    dp -= L * np.round(dp / L)
    assert np.abs(dp).max() < 1e-12
    assert np.abs(vel - d["run_vel"].reshape(-1, 3)).max() < 1e-11


def test_oracle_edge_cases(oracle_lib):
    """Ragged/edge inputs: one atom (no pairs), two atoms across the boundary,
    an atom exactly on the upper face, and the all_atom_test list."""
    O = oracle_lib
    from caviar_b200 import workloads as W
    s = W.fcc_lattice(3, 0.8442, 0.5, seed=1)
    one = s.copy()
    one.pos, one.vel, one.type = s.pos[:1], s.vel[:1], s.type[:1]
    o = O.Oracle(one)
    o.setup()
    assert o.pairs().shape == (0, 5)
    assert np.all(o.state()[2] == 0)
    two = s.copy()
    L = float(s.box[0])
    two.pos = np.array([[0.5, 1.0, 1.0], [L - 0.5, 1.0, 1.0]])
    two.vel = np.zeros((2, 3))
    two.type = np.zeros(2, np.int32)
    o = O.Oracle(two)
    o.setup()
    p = o.pairs()
    assert p.tolist() == [[0, 1, -1, 0, 0]]
    _, _, acc = o.state()
    assert acc[0, 0] > 0 and acc[1, 0] < 0 and abs(acc[0, 0] + acc[1, 0]) < 1e-12 * abs(acc[0, 0])
    face = two.copy()
    face.pos = np.array([[L, 1.0, 1.0], [L - 1.0, 1.0, 1.0]])
    o = O.Oracle(face)
    o.setup()
    assert o.pairs().shape[0] == 1


@pytest.mark.reference
def test_live_reference_matches_oracle(oracle_lib):
    """When the reference harness is built here, run it live on a fresh seed."""
    O = oracle_lib
    if not O.harness_available():
        pytest.skip("reference harness not built")
    from caviar_b200 import workloads as W
    s = W.random_ions(300, 14.0, seed=99, rc=4.5, kmax=3, alpha=0.7)
    ref = O.run_reference(s, "forces")
    o = O.Oracle(s)
    o.setup()
    assert np.array_equal(o.state()[2], ref["acc"])
    assert np.array_equal(o.pairs(), ref["pairs"])


def _jump_system():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN_DIR, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    return mg.jump_system()


def test_jump_tol_matches_reference(oracle_lib):
    """lj jump_tol (lj.cpp:118-127, 423-432): the restatement's clamp gives the
    unmodified reference's forces and virial bit for bit on a fluid with close
    pairs (tests/golden/ref_ljjump500.npz)."""
    d = np.load(os.path.join(GOLDEN_DIR, "ref_ljjump500.npz"))
    s = _jump_system()
    assert np.array_equal(s.pos, d["pos"]) and s.lj.jump_tol == float(d["jump_tol"])
    o = oracle_lib.Oracle(s)
    o.setup()
    assert np.array_equal(o.state()[2], d["acc"])
    assert o.energy()["virial"] == float(d["virial"])


def test_all_atom_test_matches_reference(oracle_lib):
    """neighborlist all_atom_test (neighborlist.cpp:161-191): the restatement's
    list (every owned pair, every ghost image) and forces equal the unmodified
    reference's (tests/golden/ref_allatom300.npz), and so does a 10-step run
    under the reference's rebuild trigger."""
    import hashlib
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN_DIR, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    d = np.load(os.path.join(GOLDEN_DIR, "ref_allatom300.npz"))
    s = mg.all_atom_system()
    o = oracle_lib.Oracle(s, all_atom_test=True)
    o.setup()
    p = o.pairs()
    assert p.shape[0] == int(d["npairs"])
    assert hashlib.sha256(np.ascontiguousarray(p, dtype="<i4").tobytes()).hexdigest() == str(d["pairs_sha256"])
    assert np.array_equal(o.state()[2], d["acc"])
    o = oracle_lib.Oracle(s, all_atom_test=True, policy=oracle_lib.POLICY_REFERENCE)
    o.setup()
    o.step(int(d["run_steps"]))
    assert np.array_equal(o.state()[0], d["run_pos"])
