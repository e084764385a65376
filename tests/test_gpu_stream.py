"""RK4 and adjoint on lattices one CTA cannot hold: streamed stages (rk_stream.cuh) and, where a
thread-block cluster holds the lattice, the cluster kernel (rk4_cluster.cuh).

Each RK4 stage is one launch over (cell tile, trajectory).  Same tolerances as
the resident path: states <= 1e-10, magnetisations / energy rows <= 1e-12
absolute; adjoint vs the FP64 tangent-linear oracle <= 1e-9 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R111 = np.ones(3) / np.sqrt(3.0)
TOL_S = 1e-10
TOL_M = 1e-12


@pytest.fixture(scope="module")
def api(native):
    from classical_mcmc_spin_b200 import gpu_api
    return gpu_api


def _spins(n, seed):
    from classical_mcmc_spin_b200.states import random_unit_spins
    return random_unit_spins(n, seed).ravel()


def _streamed(h):
    """True when no resident variant holds the handle's lattice."""
    return all(not fits for _, _, fits in h.variants())


def _default(h):
    """The variant a handle uses by default: the first that fits."""
    return next(i for i, _, fits in h.variants() if fits)


@pytest.mark.parametrize("L,streamed", [(64, True), (48, False)])
def test_batch_pump_probe_matches_oracle(api, oracle, L, streamed):
    """Per-trajectory pulse pairs on lattices one CTA cannot hold: Kitaev 64x64 (8192 spins, streamed
    stages) and 48x48 (4608 spins, one trajectory per 4-CTA cluster)."""
    from classical_mcmc_spin_b200.lattice import Lattice
    lat = Lattice.kitaev(L, L, 1)
    o = oracle.OracleLattice.kitaev(L, L, 1)
    h = lat.to_gpu()
    assert _streamed(h) == streamed
    if not streamed:
        assert h.variants()[h.get_variant() if h.get_variant() >= 0 else _default(h)][1].startswith("rk4_cluster")
    s0 = _spins(lat.lattice_size, 21)
    fin = np.tile(R111, 2)
    fd = lat.rotate_pulse(fin, fin)
    t1 = [0.0, 0.0, 0.0, 0.3]
    t2 = [0.0, 0.4, 0.4, 0.8]
    a1 = [0.5, 0.0, 0.5, 0.5]
    a2 = [0.0, 0.5, 0.5, 0.5]
    nsteps = 120
    obs, final = api.run_batch(h, s0, nsteps, 0.01, T0=-0.5, t1=t1, t2=t2, a1=a1, a2=a2, d1=fd[:6], d2=fd[6:],
                               width=0.5, freq=0.0, shared_initial=True)
    B = len(t1)
    st, oobs = oracle_batch(o, np.tile(s0, (B, 1)), t1, t2, a1, a2, fin, nsteps)
    assert obs.shape == (B, nsteps + 1, 10)
    assert np.abs(obs[:, :, :9] - oobs[:, :, :9]).max() <= TOL_M
    assert np.abs(obs[:, :, 9] - oobs[:, :, 9]).max() <= TOL_M
    assert np.abs(final - st).max() <= TOL_S


def oracle_batch(o, states, t1, t2, a1, a2, fin, nsteps):
    return o.batch_rk4(states, t1, t2, np.array(a1) / 0.5, np.array(a2) / 0.5, 0.5, 0.5, 0.0, fin, fin, -0.5, 0.01,
                       nsteps)


@pytest.mark.parametrize("L,streamed", [(10, True), (8, False)])
def test_pyrochlore_integrate_with_states(api, oracle, L, streamed):
    """Pyrochlore with a [111] field on 10^3 conventional cells (16000 spins, streamed) and 8^3 cells
    (8192 spins, 4-CTA cluster): rows, saved states, final state."""
    from classical_mcmc_spin_b200.lattice import Lattice
    kw = dict(h=0.2, Jzz=1.0, Jpm=0.05, Jpmpm=0.02)
    lat = Lattice.pyrochlore_non_kramer(L, L, L, field_direction=R111, cubic=True, **kw)
    o = oracle.OracleLattice.pyrochlore_nk(L, L, L, direction=R111, cubic=True, **kw)
    h = lat.to_gpu()
    assert _streamed(h) == streamed
    s0 = _spins(lat.lattice_size, 22)
    api.set_gpu_spins(h, s0)
    traj, obs, times = api.integrate_gpu(h, 0.0, 0.4975, 0.005, 10, "rk4", with_states=True)
    rows, fin = o.md_rk4(s0, 0.0, 0.4975, 0.005, 10, gpu_loop=True)
    assert len(rows) == len(obs) == len(traj)
    np.testing.assert_array_equal(times, rows[:, 0])
    np.testing.assert_array_equal(traj[0][1], s0)
    assert np.abs(obs[:, :9] - rows[:, 1:10]).max() <= TOL_M
    assert np.abs(obs[:, 9] - rows[:, 10]).max() <= TOL_M
    assert np.abs(traj[-1][1] - fin).max() <= TOL_S
    assert np.abs(api.get_gpu_spins(h) - fin).max() <= TOL_S


@pytest.mark.parametrize("path", ["streamed", "auto"])
def test_streamed_adjoint_kitaev_matches_tlm(native, oracle, path):
    """24x24 honeycomb (576 cells: 5 tiles of 128), two trajectories: streamed forward, recompute and VJP,
    and the resident kernel ("auto": one 576-thread CTA per trajectory)."""
    from classical_mcmc_spin_b200 import adjoint as adj
    theta = np.array([-1.0, 0.25, -0.02, 0.05, 0.1])
    build = lambda th: adj.kitaev_lattice(th, 24, 24)
    lat = build(theta)
    h = lat.to_gpu()
    B, S, dt = 2, 40, 0.01
    states = np.stack([_spins(lat.lattice_size, 90 + b) for b in range(B)])
    targets = np.random.default_rng(9).normal(scale=0.05, size=(B, S + 1, 3))
    loss, grad, mloc = adj.adjoint_rk4(h, adj.basis_lattices(build, 5), states, 0.0, dt, S, targets,
                                       checkpoint_every=7, path=path)
    ob = lambda th: oracle.OracleLattice.kitaev(24, 24, 1, h=th[4], direction=(0, 1, 0), K=th[0], Gamma=th[1],
                                                Gammap=th[2], J=th[3])
    base, basis = ob(theta), [ob(e) for e in np.eye(5)]
    for b in range(B):
        lt, gt = oracle.loss_grad_tlm(base, basis, states[b], 0.0, dt, S, targets[b])
        assert abs(loss[b] - lt) <= 1e-12 * max(1.0, abs(lt))
        np.testing.assert_allclose(grad[b], gt, rtol=1e-9, atol=1e-12)
    # forward-only loss is the same forward
    lf, _, mf = adj.adjoint_rk4(h, [], states, 0.0, dt, S, targets, forward_only=True, path=path)
    np.testing.assert_array_equal(lf, loss)
    np.testing.assert_array_equal(mf, mloc)


@pytest.mark.parametrize("path", ["streamed", "auto"])
def test_streamed_adjoint_pyrochlore_matches_tlm(native, oracle, path):
    """Pyrochlore 5^3 conventional cells (2000 spins, 500 cells: 8 tiles of 64) with a [111] field;
    "auto" runs the resident kernel on a 2-CTA cluster."""
    from classical_mcmc_spin_b200 import adjoint as adj
    theta = np.array([1.0, 0.05, 0.02, 0.2])
    build = lambda th: adj.pyrochlore_lattice(th, 5, 5, 5, cubic=True)
    lat = build(theta)
    h = lat.to_gpu()
    S, dt = 30, 0.005
    states = _spins(lat.lattice_size, 91)[None, :]
    targets = np.random.default_rng(10).normal(scale=0.05, size=(1, S + 1, 3))
    loss, grad, _ = adj.adjoint_rk4(h, adj.basis_lattices(build, 4), states, 0.0, dt, S, targets,
                                    checkpoint_every=4, path=path)
    ob = lambda th: oracle.OracleLattice.pyrochlore_nk(5, 5, 5, h=th[3], direction=R111, cubic=True, Jzz=th[0],
                                                       Jpm=th[1], Jpmpm=th[2])
    lt, gt = oracle.loss_grad_tlm(ob(theta), [ob(e) for e in np.eye(4)], states[0], 0.0, dt, S, targets[0])
    assert abs(loss[0] - lt) <= 1e-12 * max(1.0, abs(lt))
    np.testing.assert_allclose(grad[0], gt, rtol=1e-9, atol=1e-12)


def test_streamed_graph_replay_matches_direct_launches_and_oracle(api, oracle):
    """Kitaev 64x64 (streamed), 300 steps under a two-pulse drive: two replays of the captured 128-step
    chunk plus 44 direct steps give the same bits as launching every stage directly, and the oracle's
    trajectory; a second call with other pulses rebuilds the graph (different launch parameters)."""
    from classical_mcmc_spin_b200.lattice import Lattice
    lat = Lattice.kitaev(64, 64, 1)
    o = oracle.OracleLattice.kitaev(64, 64, 1)
    h = lat.to_gpu()
    assert _streamed(h)
    s0 = _spins(lat.lattice_size, 23)
    fin = np.tile(R111, 2)
    fd = lat.rotate_pulse(fin, fin)
    nsteps = 300
    for t2 in ([0.0, 0.6], [0.9, 1.3]):
        kw = dict(T0=-0.5, t1=[0.0, 0.2], t2=t2, a1=[0.5, 0.5], a2=[0.0, 0.5], d1=fd[:6], d2=fd[6:], width=0.5,
                  freq=0.0, shared_initial=True)
        h.set_graphs(True)
        og, fg = api.run_batch(h, s0, nsteps, 0.01, **kw)
        h.set_graphs(False)
        od, fdir = api.run_batch(h, s0, nsteps, 0.01, **kw)
        np.testing.assert_array_equal(og, od)
        np.testing.assert_array_equal(fg, fdir)
        st, oobs = oracle_batch(o, np.tile(s0, (2, 1)), kw["t1"], t2, kw["a1"], kw["a2"], fin, nsteps)
        assert np.abs(og[:, :, :9] - oobs[:, :, :9]).max() <= TOL_M
        assert np.abs(og[:, :, 9] - oobs[:, :, 9]).max() <= TOL_M
        assert np.abs(fg - st).max() <= TOL_S
    h.close()
