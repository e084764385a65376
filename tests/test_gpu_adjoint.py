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


@pytest.mark.parametrize("path", ["auto", "global", "streamed"])
def test_kitaev_adjoint_matches_tlm_and_fd(adj, oracle, path):
    """4x4 honeycomb, three trajectories; "auto" runs the resident kernel (one CTA per trajectory)."""
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
                                       checkpoint_every=13, path=path)
    ob = lambda th: oracle.OracleLattice.kitaev(d1, d2, 1, h=th[4], direction=(0, 1, 0), K=th[0], Gamma=th[1],
                                                Gammap=th[2], J=th[3])
    base = ob(theta)
    basis = [ob(e) for e in np.eye(5)]
    for b in range(B):
        lt, gt = oracle.loss_grad_tlm(base, basis, states[b], 0.0, dt, S, targets[b])
        assert abs(loss[b] - lt) <= 1e-12 * max(1.0, abs(lt))
        np.testing.assert_allclose(grad[b], gt, rtol=1e-9, atol=1e-12)
    if path != "auto":
        return
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


@pytest.mark.parametrize("path", ["auto", "global"])
def test_pyrochlore_adjoint_matches_tlm(adj, oracle, path):
    theta = np.array([1.0, 0.05, 0.02, 0.2])
    build = lambda th: adj.pyrochlore_lattice(th, 1, 1, 1, cubic=True)
    lat = build(theta)
    h = lat.to_gpu()
    S, dt = 80, 0.005
    states = _spins(lat.lattice_size, 70)[None, :]
    targets = np.random.default_rng(6).normal(scale=0.05, size=(1, S + 1, 3))
    loss, grad, _ = adj.adjoint_rk4(h, adj.basis_lattices(build, 4), states, 0.0, dt, S, targets, path=path)
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


def test_resident_adjoint_48x48_cluster_driven(adj, oracle):
    """48x48 honeycomb (2304 cells: one trajectory per 4-CTA cluster) under a two-pulse drive, a field
    and all five parameters: the resident adjoint against the tangent-linear oracle, and against the
    streamed path (the same derivative, another summation order)."""
    theta = np.array([-1.0, 0.25, -0.02, 0.05, 0.1])
    build = lambda th: adj.kitaev_lattice(th, 48, 48)
    lat = build(theta)
    h = lat.to_gpu()
    fin = np.tile(np.ones(3) / np.sqrt(3.0), 2)
    from classical_mcmc_spin_b200 import gpu_api
    gpu_api.set_gpu_pulse(h, lat.rotate_pulse(fin, fin), 0.4, 0.05, 0.8, 0.06, 0.15)
    B, S, dt = 2, 30, 0.01
    states = np.stack([_spins(lat.lattice_size, 95 + b) for b in range(B)])
    targets = np.random.default_rng(11).normal(scale=0.05, size=(B, S + 1, 3))
    dps = adj.basis_lattices(build, 5)
    loss, grad, mloc = adj.adjoint_rk4(h, dps, states, 0.0, dt, S, targets, checkpoint_every=7, path="resident")
    ls, gs, ms = adj.adjoint_rk4(h, dps, states, 0.0, dt, S, targets, checkpoint_every=7, path="streamed")
    np.testing.assert_allclose(mloc, ms, rtol=0, atol=1e-13)
    np.testing.assert_allclose(loss, ls, rtol=1e-12)
    np.testing.assert_allclose(grad, gs, rtol=1e-10, atol=1e-13)
    ob = lambda th: oracle.OracleLattice.kitaev(48, 48, 1, h=th[4], direction=(0, 1, 0), K=th[0], Gamma=th[1],
                                                Gammap=th[2], J=th[3])
    base, basis = ob(theta), [ob(e) for e in np.eye(5)]
    base.set_pulse(fin, 0.06, fin, 0.15, 0.4, 0.05, 0.8)
    for b in range(B):
        lt, gt = oracle.loss_grad_tlm(base, basis, states[b], 0.0, dt, S, targets[b])
        assert abs(loss[b] - lt) <= 1e-12 * max(1.0, abs(lt))
        np.testing.assert_allclose(grad[b], gt, rtol=1e-9, atol=1e-12)
    lf, _, mf = adj.adjoint_rk4(h, [], states, 0.0, dt, S, targets, forward_only=True)
    np.testing.assert_array_equal(lf, loss)
    np.testing.assert_array_equal(mf, mloc)
