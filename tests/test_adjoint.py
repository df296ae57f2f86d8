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


# ------------------------------------------------------------------ GPU

def gpu_engine(abi, s, prec):
    return abi.Adjoint.from_system(s, prec)


def medium_system():
    # 256 atoms (FCC 4^3), L = 6.72; rc_lj 2.5, rc_r 3.3 (< L/2), alpha 0.9, k_max 5
    return W.adjoint_mixture(ncell=4, alpha=0.9, rc_r=3.3, kmax=5)


def rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [(1, 1e-11), (0, 1e-5)])
@pytest.mark.parametrize("which", ["medium", "mixture4000"])
def test_gpu_forces_energy_dU(cuda_lib, oracle_lib, prec, tol, which):
    s = medium_system() if which == "medium" else W.adjoint_mixture()
    a = gpu_engine(cuda_lib, s, prec)
    f, e, dU = a.forces()
    o = oracle_lib.AdjOracle(s)
    f0, e0, dU0 = o.forces(s.pos)
    assert rel(f, f0) < tol
    for k in range(4):
        assert abs(e[k] - e0[k]) <= tol * max(1.0, abs(e0[k])), (k, e[k], e0[k])
    for k in ("eps", "sigma", "charge"):
        assert rel(dU[k], dU0[k]) < tol, k


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [(1, 1e-10), (0, 1e-5)])
def test_gpu_force_vjp(cuda_lib, oracle_lib, prec, tol):
    s = medium_system()
    a = gpu_engine(cuda_lib, s, prec)
    u = np.random.default_rng(3).normal(size=s.pos.shape)
    w, g = a.force_vjp(u)
    w0, g0 = oracle_lib.AdjOracle(s).force_vjp(s.pos, u)
    assert rel(w, w0) < tol
    for k in ("eps", "sigma", "charge"):
        assert rel(g[k], g0[k]) < tol, k


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [(1, 1e-9), (0, 1e-4)])
def test_gpu_trajectory_gradient_matches_oracle(cuda_lib, oracle_lib, prec, tol):
    s = medium_system()
    M, K = 40, 15
    J0, g0 = oracle_lib.AdjOracle(s).loss_grad(s.pos, s.vel, M, K)
    a = gpu_engine(cuda_lib, s, prec)
    J, g = a.loss_grad(M, K)
    assert abs(J - J0) <= tol * abs(J0)
    for k in ("pos", "vel", "eps", "sigma", "charge"):
        assert rel(g[k], g0[k]) < tol, (k, rel(g[k], g0[k]))
    assert abs(a.loss(M) - J) <= 1e-12 * abs(J)


@pytest.mark.gpu
def test_gpu_mixture4000_gradient_matches_fd(cuda_lib):
    """The 4000-atom mixture, 500 steps (dt 0.002), checkpoints every 50: the
    mixed-precision and FP64 adjoint gradients against central differences
    (h = 1e-4) of the FP64 GPU loss, along a random position direction, a
    random velocity direction and every parameter."""
    s = W.adjoint_mixture()
    M, K = 500, 50
    mixed = gpu_engine(cuda_lib, s, 0)
    J_m, g_m = mixed.loss_grad(M, K)
    f64 = gpu_engine(cuda_lib, s, 1)
    J_d, g_d = f64.loss_grad(M, K)
    assert abs(J_m - J_d) <= 1e-5 * abs(J_d)
    rng = np.random.default_rng(11)

    def loss_at(pos, vel, eps, sig, q):
        f64.set_params(q, eps, sig, s.rc_lj, s.alpha, s.rc_r, s.kmax, s.k_e, s.dt)
        f64.set_state(pos, vel, s.type)
        return f64.loss(M)

    checks = []
    for which in ("pos", "vel"):
        dirn = rng.normal(size=s.pos.shape)
        dirn /= np.linalg.norm(dirn)
        vals = []
        for sg in (1, -1):
            p = s.pos + sg * H * dirn if which == "pos" else s.pos
            v = s.vel + sg * H * dirn if which == "vel" else s.vel
            vals.append(loss_at(p, v, s.epsilon, s.sigma, s.charge))
        fd = (vals[0] - vals[1]) / (2 * H)
        checks.append((which, float(np.sum(g_d[which] * dirn)), float(np.sum(g_m[which] * dirn)), fd,
                       np.linalg.norm(g_d[which])))
    for name, idx in PARAMS:
        vals = []
        for sg in (1, -1):
            m = perturbed(s, name, idx, sg * H)
            vals.append(loss_at(s.pos, s.vel, m["eps"], m["sigma"], m["charge"]))
        fd = (vals[0] - vals[1]) / (2 * H)
        checks.append((name + str(idx), float(g_d[name][idx]), float(g_m[name][idx]), fd, np.abs(g_d[name]).max()))
    for name, gd, gm, fd, scale in checks:
        assert abs(gd - fd) <= 1e-5 * scale + 1e-5 * abs(fd), (name, gd, fd)
        assert abs(gm - fd) <= 1e-4 * scale + 1e-4 * abs(fd), (name, gm, fd)


@pytest.mark.gpu
def test_torch_autograd_binding(cuda_lib):
    import torch
    from torch_adjoint import Engine, Forces, TrajectoryLoss, sym2
    s = small_system()
    eng = Engine(s, precision=1, nsteps=8, checkpoint_every=3)
    pos = torch.tensor(s.pos, requires_grad=True)
    vel = torch.tensor(s.vel, requires_grad=True)
    ev = torch.tensor([s.epsilon[0, 0], s.epsilon[0, 1], s.epsilon[1, 1]], requires_grad=True)
    sv = torch.tensor([s.sigma[0, 0], s.sigma[0, 1], s.sigma[1, 1]], requires_grad=True)
    q = torch.tensor(s.charge, requires_grad=True)
    J = TrajectoryLoss.apply(pos, vel, sym2(ev), sym2(sv), q, eng)
    J.backward()
    J_ref, g = eng.a.loss_grad(8, 3)
    assert abs(J.item() - J_ref) <= 1e-12 * abs(J_ref)
    assert np.allclose(pos.grad.numpy(), g["pos"], rtol=1e-12, atol=0)
    assert np.allclose(vel.grad.numpy(), g["vel"], rtol=1e-12, atol=0)
    assert np.allclose(ev.grad.numpy(), [g["eps"][0, 0], g["eps"][0, 1], g["eps"][1, 1]], rtol=1e-12, atol=0)
    assert np.allclose(q.grad.numpy(), g["charge"], rtol=1e-12, atol=0)
    # Forces: the full Jacobian by finite differences against the VJP kernel (FP64)
    args = (torch.tensor(s.pos, requires_grad=True), ev.detach().clone().requires_grad_(),
            sv.detach().clone().requires_grad_(), q.detach().clone().requires_grad_())
    assert torch.autograd.gradcheck(lambda p, e, sg, qq: Forces.apply(p, sym2(e), sym2(sg), qq, eng), args,
                                    eps=1e-6, atol=1e-5, rtol=1e-4)
