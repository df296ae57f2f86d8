"""CPU checks that the seeded workload generators produce the systems the
benchmark and the parity tests are defined on: atom counts, densities,
temperatures (2 KE / (3N - 3) with the centre-of-mass motion removed, the
reference's periodic degrees of freedom), charges, cutoffs and spacing."""
import numpy as np
from scipy.spatial import cKDTree

from caviar_b200 import workloads as W


def _temperature(vel, mass=1.0):
    return float(mass * np.sum(vel * vel) / (3 * len(vel) - 3))


def test_lj_1m_fluid():
    s = W.config_lj_1m(seed=3)
    assert s.n == 1_048_576
    L = s.box
    assert np.allclose(L, L[0]) and abs(s.n / np.prod(L) - 0.8442) < 1e-12
    assert abs(_temperature(s.vel) - 0.72) < 1e-10
    assert np.abs(s.vel.sum(axis=0)).max() < 1e-8
    assert (s.pos >= 0).all() and (s.pos < L).all()
    assert s.cutoff == 2.5 and abs(s.cutoff * s.coef - 2.8) < 1e-12  # rl = rc + skin 0.3
    assert s.ghost_cutoff >= s.cutoff * s.coef and s.ghost_cutoff <= 0.5 * L.min()


def test_lj_4000_same_recipe():
    s = W.config_lj_4000(seed=1)
    assert s.n == 4000 and abs(s.n / np.prod(s.box) - 0.8442) < 1e-12
    assert abs(_temperature(s.vel) - 0.72) < 1e-10


def test_ions_8000():
    s = W.config_ions_8000(seed=2)
    assert s.n == 8000 and np.allclose(s.box, 40.0)
    q = s.charge[s.type]
    assert q.sum() == 0.0 and (np.abs(q) == 1.0).all()
    assert s.ewald_r.alpha == 0.3 and s.ewald_k.alpha == 0.3 and s.ewald_k.kmax == (8, 8, 8)
    assert s.cutoff == 10.0 and abs(s.cutoff * s.coef - 10.3) < 1e-12
    # non-overlapping: no pair closer than 0.9 sigma under the minimum image
    tree = cKDTree(s.pos, boxsize=40.0)
    assert len(tree.query_pairs(0.9 * (1 - 1e-12))) == 0
    assert np.abs(s.vel.sum(axis=0)).max() < 1e-9


def test_replica_batch():
    b = W.replica_batch()
    assert len(b.n) == 1024 and b.n.min() >= 64 and b.n.max() <= 2048
    assert np.allclose(b.n / b.box ** 3, 0.8)
    assert (b.temperature >= 0.7).all() and (b.temperature <= 1.5).all()
    off = b.offsets
    for r in (0, 17, 511, 1023):
        t = b.type[off[r]:off[r + 1]]
        q = b.charge[t]
        assert q.sum() == 0.0
        assert abs(np.count_nonzero(q) - b.n[r] / 2) <= 2  # half the atoms charged
        v = b.vel[off[r]:off[r + 1]]
        assert abs(_temperature(v) - b.temperature[r]) < 1e-10
        p = b.pos[off[r]:off[r + 1]]
        assert (p >= 0).all() and (p < b.box[r]).all()
    assert np.allclose(b.rc_r, b.box / 2) and np.allclose(b.rc_lj, np.minimum(2.5, b.box / 2))
    assert b.alpha == 0.35 and b.kmax == 6


def test_adjoint_mixture():
    s = W.adjoint_mixture()
    assert len(s.pos) == 4000 and abs(s.box - 16.796) < 1e-3
    assert np.count_nonzero(s.type == 0) == 2000
    assert np.allclose(s.epsilon, [[1.0, 0.75], [0.75, 0.5]]) and np.allclose(s.sigma, [[1.0, 0.94], [0.94, 0.88]])
    assert np.allclose(s.charge, [0.5, -0.5]) and s.dt == 0.002
