"""Trajectory adjoint: gradient of J = (1/M) sum_{t=1..M} U(r_t) over M
velocity-Verlet steps w.r.t. initial positions, velocities, eps/sigma per type
pair and per-type charges.

The reference has no gradients, so parity is pinned by central finite
differences (h = 1e-4) of FP64 forwards:
CPU: the FP64 restatement (oracle/adjoint.c) -- its force VJP, dU/dtheta and
  checkpointed trajectory gradient -- against its own FD.
GPU: the CUDA adjoint (cvr_adj_*) against the restatement (forces, VJP,
  trajectory gradient) and against FD of the GPU's own FP64 forward at the
  4000-atom mixture, 500 steps, checkpoints every 50.
"""
import numpy as np
import pytest

from caviar_b200 import workloads as W

H = 1e-4


def small_system():
    # 32 atoms, L = 3.36: every cutoff is L/2; alpha 1.0, k_max 3
    return W.adjoint_mixture(ncell=2, alpha=1.0, kmax=3)


def perturbed(s, name, idx, delta):
    m = {"eps": s.epsilon.copy(), "sigma": s.sigma.copy(), "charge": s.charge.copy()}
    x = m[name]
    x[idx] += delta
    if len(idx) == 2 and idx[0] != idx[1]:
        x[idx[::-1]] += delta
    return m


PARAMS = [("eps", (0, 0)), ("eps", (0, 1)), ("eps", (1, 1)), ("sigma", (0, 0)), ("sigma", (0, 1)),
          ("sigma", (1, 1)), ("charge", (0,)), ("charge", (1,))]


def close(a, b, rel, floor=1e-9):
    return abs(a - b) <= rel * max(abs(a), abs(b)) + floor


def test_oracle_force_vjp_matches_fd(oracle_lib):
    s = small_system()
    a = oracle_lib.AdjOracle(s)
    u = np.random.default_rng(0).normal(size=s.pos.shape)
    w, g = a.force_vjp(s.pos, u)
    h = 1e-5
    for i, d in [(0, 0), (5, 2), (17, 1), (31, 0)]:
        p1, p2 = s.pos.copy(), s.pos.copy()
        p1[i, d] += h
        p2[i, d] -= h
        fd = (np.sum(u * a.forces(p1)[0]) - np.sum(u * a.forces(p2)[0])) / (2 * h)
        assert close(w[i, d], fd, 1e-6), (i, d, w[i, d], fd)
    _, _, dU = a.forces(s.pos)
    for name, idx in PARAMS:
        vals = []
        for sg in (1, -1):
            m = perturbed(s, name, idx, sg * h)
            a.set_params(m["eps"], m["sigma"], m["charge"])
            F, e, _ = a.forces(s.pos)
            vals.append((np.sum(u * F), e.sum()))
        a.set_params(s.epsilon, s.sigma, s.charge)
        assert close(g[name][idx], (vals[0][0] - vals[1][0]) / (2 * h), 1e-6), (name, idx)
        assert close(dU[name][idx], (vals[0][1] - vals[1][1]) / (2 * h), 1e-6), (name, idx)


def test_oracle_forces_are_minus_energy_gradient(oracle_lib):
    s = small_system()
    a = oracle_lib.AdjOracle(s)
    F, _, _ = a.forces(s.pos)
    h = 1e-5
    for i, d in [(3, 0), (9, 1), (20, 2)]:
        p1, p2 = s.pos.copy(), s.pos.copy()
        p1[i, d] += h
        p2[i, d] -= h
        fd = -(a.forces(p1)[1].sum() - a.forces(p2)[1].sum()) / (2 * h)
        assert close(F[i, d], fd, 1e-6)


@pytest.mark.parametrize("M,K", [(20, 6), (12, 12), (9, 1)])
def test_oracle_trajectory_gradient_matches_fd(oracle_lib, M, K):
    s = small_system()
    a = oracle_lib.AdjOracle(s)
    J, g = a.loss_grad(s.pos, s.vel, M, K)
    assert close(J, a.loss(s.pos, s.vel, M), 1e-13)
    for i, d in [(0, 0), (7, 1), (31, 2)]:
        for which in ("pos", "vel"):
            p1, v1, p2, v2 = s.pos.copy(), s.vel.copy(), s.pos.copy(), s.vel.copy()
            (p1 if which == "pos" else v1)[i, d] += H
            (p2 if which == "pos" else v2)[i, d] -= H
            fd = (a.loss(p1, v1, M) - a.loss(p2, v2, M)) / (2 * H)
            assert close(g[which][i, d], fd, 1e-5, 1e-7), (which, i, d, g[which][i, d], fd)
    # FD truncation error is O(h^2) (about 4e-5 on sigma at h = 1e-4, where
    # U ~ sigma^12): compare at h = 1e-4 to 1e-5 of the class's largest
    # gradient, and the Richardson extrapolation of h and h/2 (O(h^4)) tightly.
    for name, idx in PARAMS:
        fd = []
        for h in (H, H / 2):
            vals = []
            for sg in (1, -1):
                m = perturbed(s, name, idx, sg * h)
                a.set_params(m["eps"], m["sigma"], m["charge"])
                vals.append(a.loss(s.pos, s.vel, M))
            a.set_params(s.epsilon, s.sigma, s.charge)
            fd.append((vals[0] - vals[1]) / (2 * h))
        scale = max(1.0, np.abs(g[name]).max())
        rich = (4 * fd[1] - fd[0]) / 3
        assert abs(g[name][idx] - fd[0]) <= 1e-5 * scale, (name, idx, g[name][idx], fd)
        assert abs(g[name][idx] - rich) <= 1e-7 * scale, (name, idx, g[name][idx], rich)


def test_mixture_generator():
    s = W.adjoint_mixture()
    assert s.pos.shape == (4000, 3) and abs(s.box - 16.796) < 1e-3
    assert np.count_nonzero(s.type == 0) == 2000
    assert np.all((s.pos >= 0) & (s.pos < s.box))
    assert s.rc_r <= s.box / 2 and s.rc_lj <= s.box / 2
    assert s.epsilon[0, 1] == 0.75 and s.sigma[1, 1] == 0.88 and abs(s.sigma[0, 1] - 0.94) < 1e-15
