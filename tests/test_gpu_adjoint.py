"""Discrete adjoint vs the FP64 tangent-linear reference (oracle) and central finite differences.

Tolerances: adjoint vs tangent-linear (both exact derivatives of the same
discrete map, FP64): <= 1e-9 relative per component; adjoint vs central FD
(eps = 1e-5, GPU forward passes): <= 1e-6 relative (the task's gate).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def adj(native):
    from classical_mcmc_spin_b200 import adjoint
    return adjoint


def _spins(n, seed):
    from classical_mcmc_spin_b200.states import random_unit_spins
    return random_unit_spins(n, seed).ravel()


def test_kitaev_adjoint_matches_tlm_and_fd(adj, oracle):
    theta = np.array([-1.0, 0.25, -0.02, 0.0, 0.0])
    d1 = d2 = 4
    S, dt = 150, 0.01
    build = lambda th: adj.kitaev_lattice(th, d1, d2)
    lat = build(theta)
    h = lat.to_gpu()
    B = 3
    states = np.stack([_spins(lat.lattice_size, 60 + b) for b in range(B)])
    rng = np.random.default_rng(5)
    targets = rng.normal(scale=0.05, size=(B, S + 1, 3))
    loss, grad, mloc = adj.adjoint_rk4(h, adj.basis_lattices(build, 5), states, 0.0, dt, S, targets,
                                       checkpoint_every=13)
    ob = lambda th: oracle.OracleLattice.kitaev(d1, d2, 1, h=th[4], direction=(0, 1, 0), K=th[0], Gamma=th[1],
                                                Gammap=th[2], J=th[3])
    base = ob(theta)
    basis = [ob(e) for e in np.eye(5)]
    for b in range(B):
        lt, gt = oracle.loss_grad_tlm(base, basis, states[b], 0.0, dt, S, targets[b])
        assert abs(loss[b] - lt) <= 1e-12 * max(1.0, abs(lt))
        np.testing.assert_allclose(grad[b], gt, rtol=1e-9, atol=1e-12)
    # central finite differences of the GPU forward pass
    eps = 1e-5
    for q in range(5):
        tp, tm = theta.copy(), theta.copy()
        tp[q] += eps
        tm[q] -= eps
        hp, hm = build(tp).to_gpu(), build(tm).to_gpu()
        lp, _, _ = adj.adjoint_rk4(hp, [], states, 0.0, dt, S, targets, forward_only=True)
        lm, _, _ = adj.adjoint_rk4(hm, [], states, 0.0, dt, S, targets, forward_only=True)
        fd = (lp - lm) / (2 * eps)
        np.testing.assert_allclose(grad[:, q], fd, rtol=1e-6, atol=1e-9)


def test_pyrochlore_adjoint_matches_tlm(adj, oracle):
    theta = np.array([1.0, 0.05, 0.02, 0.2])
    build = lambda th: adj.pyrochlore_lattice(th, 1, 1, 1, cubic=True)
    lat = build(theta)
    h = lat.to_gpu()
    S, dt = 80, 0.005
    states = _spins(lat.lattice_size, 70)[None, :]
    targets = np.random.default_rng(6).normal(scale=0.05, size=(1, S + 1, 3))
    loss, grad, _ = adj.adjoint_rk4(h, adj.basis_lattices(build, 4), states, 0.0, dt, S, targets)
    R = np.ones(3) / np.sqrt(3.0)
    ob = lambda th: oracle.OracleLattice.pyrochlore_nk(1, 1, 1, h=th[3], direction=R, cubic=True, Jzz=th[0],
                                                       Jpm=th[1], Jpmpm=th[2])
    lt, gt = oracle.loss_grad_tlm(ob(theta), [ob(e) for e in np.eye(4)], states[0], 0.0, dt, S, targets[0])
    assert abs(loss[0] - lt) <= 1e-12 * max(1.0, abs(lt))
    np.testing.assert_allclose(grad[0], gt, rtol=1e-9, atol=1e-12)


def test_torch_autograd_function(adj):
    import torch
    theta = torch.tensor([-1.0, 0.25, -0.02, 0.0, 0.1], dtype=torch.float64, requires_grad=True)
    build = lambda th: adj.kitaev_lattice(th, 3, 3)
    lat = build(theta.detach().numpy())
    states = _spins(lat.lattice_size, 80)[None, :]
    S = 50
    targets = np.zeros((1, S + 1, 3))
    loss = adj.LLTrajectoryLoss.apply(theta, build, states, targets, 0.0, 0.01, S, 7)
    loss.backward()
    h = lat.to_gpu()
    l2, g2, _ = adj.adjoint_rk4(h, adj.basis_lattices(build, 5), states, 0.0, 0.01, S, targets, 7)
    assert abs(loss.item() - l2[0]) <= 1e-14 * max(1.0, abs(l2[0]))
    np.testing.assert_allclose(theta.grad.numpy(), g2[0], rtol=1e-12)
