"""Parity at the benchmarked workloads' own sizes and settings.

* Batched 2DCS scan (768 trajectories x 1152 spins, zigzag + sigma 0.05 tilt seed 2, T_start = -5, the scan's
  pump-only / probe-only / pump+probe pulses): the whole scan runs in one launch for 1000 RK4 steps; 24
  trajectories spread over the delays and all three pulse kinds are compared with the oracle's batched RK4
  (lattice_md.cpp:683-926 restated): max|dS| <= 1e-10 (the task's 1000-step gate), rows <= 1e-12.
* The 2DCS spectrum of a reduced but real scan (32 delays, 1152 spins, 2000 steps, the coherent window):
  M_NL and |FFT2| from the GPU rows through cmd_nonlinear_spectrum against the oracle's trajectories through
  the reader restatement (reader_honeycomb.py:459-560): 1e-6 relative (the task's spectrum gate).
* Uneven RK45 batch sizes (honeycomb L = 32, pyrochlore 6^3 and 8^3 cubic cells, tol 1e-10): accepted and
  rejected step counts identical to the oracle's controller (lattice.h:4072-4078 restated), rows <= 1e-7.
* 48x48 adjoint with the benchmark's 141-step checkpoints over 500 steps (4 segments): tangent-linear
  agreement <= 1e-9, central finite differences <= 1e-6.  Over t = 5 the derivative of the map is well
  conditioned (the chaotic growth exp(lambda t) that makes the 2x10^4-step gradient astronomically large has
  not set in).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R111 = np.ones(3) / np.sqrt(3.0)


@pytest.fixture(scope="module")
def api(native):
    from classical_mcmc_spin_b200 import gpu_api
    return gpu_api


def _scan(taus):
    t1, t2, a1, a2 = [], [], [], []
    for tau in taus:
        for (x1, x2) in ((0.5, 0.0), (0.0, 0.5), (0.5, 0.5)):
            t1.append(0.0); t2.append(tau); a1.append(x1); a2.append(x2)
    return np.array(t1), np.array(t2), np.array(a1), np.array(a2)


def _kitaev24(oracle):
    from classical_mcmc_spin_b200.lattice import Lattice
    from classical_mcmc_spin_b200.states import zigzag_honeycomb
    lat = Lattice.kitaev(24, 24, 1, K=-1.0, Gamma=0.25, Gammap=-0.02)
    o = oracle.OracleLattice.kitaev(24, 24, 1, K=-1.0, Gamma=0.25, Gammap=-0.02)
    s0 = zigzag_honeycomb(24, 24, 1, tilt_sigma=0.05, seed=2).ravel()
    return lat, o, s0


def test_config2_scan_1000_steps_matches_oracle(api, oracle):
    lat, o, s0 = _kitaev24(oracle)
    fin = np.tile(R111, 2)
    fd = lat.rotate_pulse(fin, fin)
    taus = 100.0 * np.arange(256) / 255.0
    t1, t2, a1, a2 = _scan(taus)
    B, S = len(t1), 1000
    assert B == 768
    h = lat.to_gpu()
    obs, final = api.run_batch(h, s0, S, 0.01, T0=-5.0, t1=t1, t2=t2, a1=a1, a2=a2, d1=fd[:6], d2=fd[6:],
                               width=0.5, freq=0.0, shared_initial=True)
    h.close()
    assert obs.shape == (B, S + 1, 10)
    # delays whose probe falls inside the window (tau < 5) and far outside it, every pulse kind
    ks = [0, 1, 2, 3, 5, 8, 12, 255]
    pick = [3 * k + j for k in ks for j in range(3)]
    st, oobs = o.batch_rk4(np.tile(s0, (len(pick), 1)), t1[pick], t2[pick], a1[pick] / 0.5, a2[pick] / 0.5, 0.5,
                           0.5, 0.0, fin, fin, -5.0, 0.01, S)
    assert np.abs(final[pick] - st).max() <= 1e-10
    assert np.abs(obs[pick, :, :9] - oobs[:, :, :9]).max() <= 1e-12
    assert np.abs(obs[pick, :, 9] - oobs[:, :, 9]).max() <= 1e-12
    # the driven trajectories really differ from one another inside the window
    assert np.abs(obs[3 * 1 + 2, -1, :9] - obs[3 * 12 + 2, -1, :9]).max() > 1e-6


def test_config2_batched_spectrum_matches_oracle(native, api, oracle):
    import spectra_oracle as so
    lat, o, s0 = _kitaev24(oracle)
    fin = np.tile(R111, 2)
    fd = lat.rotate_pulse(fin, fin)
    n_tau, S = 32, 2000
    taus = 10.0 * np.arange(n_tau) / (n_tau - 1)
    t1, t2, a1, a2 = _scan(taus)
    h = lat.to_gpu()
    obs, _ = api.run_batch(h, s0, S, 0.01, T0=-5.0, t1=t1, t2=t2, a1=a1, a2=a2, d1=fd[:6], d2=fd[6:],
                           width=0.5, freq=0.0, shared_initial=True, want_final=False)
    h.close()
    _, oobs = o.batch_rk4(np.tile(s0, (len(t1), 1)), t1, t2, a1 / 0.5, a2 / 0.5, 0.5, 0.5, 0.0, fin, fin, -5.0,
                          0.01, S)
    ml_g, ml_o = obs[:, :, 3:6], oobs[:, :, 3:6]            # M_local, as the reader uses
    D = native.dptr
    for c in range(3):
        M0g, M1g, M01g = (np.ascontiguousarray(ml_g[0]), np.ascontiguousarray(ml_g[1::3]),
                          np.ascontiguousarray(ml_g[2::3]))
        nl = np.zeros((n_tau, S + 1))
        sp = np.zeros((n_tau, S + 1))
        native.check(native.lib().cmd_nonlinear_spectrum(D(M0g), D(M1g), D(M01g), n_tau, S + 1, c, D(nl), D(sp)),
                     "cmd_nonlinear_spectrum")
        ref = so.compute_2d_fft(so.nonlinear_signal(ml_o[0], ml_o[1::3], ml_o[2::3], c))
        assert np.abs(ref).max() > 0
        assert np.abs(sp - ref).max() <= 1e-6 * np.abs(ref).max()


def test_config3_uneven_rk45_sizes_match_oracle_controller(api, oracle):
    """The uneven batch's largest sizes: honeycomb 32x32 (2048 spins) and pyrochlore 6^3 / 8^3 conventional
    cells (3456 / 8192 spins) in one launch, tol 1e-10 (abs = rel), dt0 = 0.01, T = 3."""
    from classical_mcmc_spin_b200.lattice import Lattice
    from classical_mcmc_spin_b200.states import random_unit_spins
    kw = dict(Jzz=1.0, Jpm=0.05, Jpmpm=0.02)
    cases = [(Lattice.kitaev(32, 32, 1, K=-1.0, Gamma=0.25, Gammap=-0.02),
              oracle.OracleLattice.kitaev(32, 32, 1, K=-1.0, Gamma=0.25, Gammap=-0.02))]
    for L in (6, 8):
        cases.append((Lattice.pyrochlore_non_kramer(L, L, L, cubic=True, **kw),
                      oracle.OracleLattice.pyrochlore_nk(L, L, L, cubic=True, **kw)))
    handles = [c[0].to_gpu() for c in cases]
    T1 = 3.0
    specs = [dict(handle=hh, state=random_unit_spins(lat.lattice_size, 300 + i).ravel(), T0=0.0, T1=T1, dt=0.01,
                  max_rows=20000) for i, ((lat, _), hh) in enumerate(zip(cases, handles))]
    out = api.run_uneven(specs, "rk45", 1e-10, 1e-10)
    for i, ((lat, o), sp) in enumerate(zip(cases, specs)):
        rows, fin, stats = out[i]
        orows, ofin, ostats = o.md_dopri5(sp["state"], 0.0, T1, 0.01, 1e-10, 1e-10)
        assert ostats[0] >= 100, ostats                    # a few hundred accepted steps
        assert stats[3] == 0 and stats[1] == ostats[0] and stats[2] == ostats[1], (i, stats, ostats)
        assert len(rows) == len(orows)
        assert np.abs(rows[:, 0] - orows[:, 0]).max() <= 1e-7
        assert np.abs(rows[:, 1:] - orows[:, 1:]).max() <= 1e-7
        assert np.abs(fin - ofin).max() <= 1e-9
    for hh in handles:
        hh.close()


def test_config4_adjoint_48x48_checkpoint141_matches_tlm_and_fd(oracle):
    from classical_mcmc_spin_b200 import adjoint as A
    from classical_mcmc_spin_b200.states import random_unit_spins
    theta = np.array([-1.0, 0.25, -0.02, 0.0, 0.0])
    theta_t = np.array([-1.0, 0.3, -0.03, 0.0, 0.1])
    build = lambda th: A.kitaev_lattice(th, 48, 48)
    lat = build(theta)
    N, B, S, dt, ckpt = lat.lattice_size, 2, 500, 0.01, 141
    h, ht = lat.to_gpu(), build(theta_t).to_gpu()
    states = np.stack([random_unit_spins(N, 4000 + b).ravel() for b in range(B)])
    _, _, target = A.adjoint_rk4(ht, [], states, 0.0, dt, S, np.zeros((B, S + 1, 3)), forward_only=True)
    loss, grad, _ = A.adjoint_rk4(h, A.basis_lattices(build, 5), states, 0.0, dt, S, target,
                                  checkpoint_every=ckpt)
    ob = lambda th: oracle.OracleLattice.kitaev(48, 48, 1, h=th[4], direction=(0, 1, 0), K=th[0], Gamma=th[1],
                                                Gammap=th[2], J=th[3])
    base, basis = ob(theta), [ob(e) for e in np.eye(5)]
    for b in range(B):
        lt, gt = oracle.loss_grad_tlm(base, basis, states[b], 0.0, dt, S, target[b])
        assert abs(loss[b] - lt) <= 1e-12 * max(1.0, abs(lt))
        np.testing.assert_allclose(grad[b], gt, rtol=1e-9, atol=1e-12 * np.abs(gt).max())
    eps = 1e-5
    for q in range(5):
        tp, tm = theta.copy(), theta.copy()
        tp[q] += eps
        tm[q] -= eps
        hp, hm = build(tp).to_gpu(), build(tm).to_gpu()
        lp, _, _ = A.adjoint_rk4(hp, [], states, 0.0, dt, S, target, forward_only=True)
        lm, _, _ = A.adjoint_rk4(hm, [], states, 0.0, dt, S, target, forward_only=True)
        hp.close()
        hm.close()
        fd = (lp - lm) / (2 * eps)
        np.testing.assert_allclose(grad[:, q], fd, rtol=1e-6, atol=1e-6 * np.abs(grad).max())
    h.close()
    ht.close()


def test_config5_adjoint_pyrochlore65536_matches_tlm_and_fd(oracle):
    """The large-lattice adjoint at its own size: pyrochlore 16^3 conventional cells (65536 spins, streamed
    kernels), parameters (Jzz, J+-, J+-+-, h along [111]) as in the benchmark's leg, 24 steps of dt = 0.005 with a
    checkpoint every 5 steps (four full segments and a partial one): loss <= 1e-12, gradient <= 1e-9 against the
    tangent-linear oracle and <= 1e-6 against central finite differences of the GPU forward."""
    from classical_mcmc_spin_b200 import adjoint as A
    from classical_mcmc_spin_b200.states import random_unit_spins
    theta = np.array([1.0, 0.05, 0.02, 0.2])
    build = lambda th: A.pyrochlore_lattice(th, 16, 16, 16, cubic=True)
    lat = build(theta)
    N, S, dt = lat.lattice_size, 24, 0.005
    assert N == 65536
    h, ht = lat.to_gpu(), build(np.array([1.0, 0.06, 0.03, 0.25])).to_gpu()
    states = random_unit_spins(N, 5000).ravel()[None, :]
    _, _, target = A.adjoint_rk4(ht, [], states, 0.0, dt, S, np.zeros((1, S + 1, 3)), forward_only=True)
    loss, grad, _ = A.adjoint_rk4(h, A.basis_lattices(build, 4), states, 0.0, dt, S, target, checkpoint_every=5)
    ob = lambda th: oracle.OracleLattice.pyrochlore_nk(16, 16, 16, h=th[3], direction=R111, cubic=True, Jzz=th[0],
                                                       Jpm=th[1], Jpmpm=th[2])
    lt, gt = oracle.loss_grad_tlm(ob(theta), [ob(e) for e in np.eye(4)], states[0], 0.0, dt, S, target[0])
    assert abs(loss[0] - lt) <= 1e-12 * max(1.0, abs(lt))
    np.testing.assert_allclose(grad[0], gt, rtol=1e-9, atol=1e-12 * np.abs(gt).max())
    eps = 1e-5
    for q in range(4):
        tp, tm = theta.copy(), theta.copy()
        tp[q] += eps
        tm[q] -= eps
        hp, hm = build(tp).to_gpu(), build(tm).to_gpu()
        lp, _, _ = A.adjoint_rk4(hp, [], states, 0.0, dt, S, target, forward_only=True)
        lm, _, _ = A.adjoint_rk4(hm, [], states, 0.0, dt, S, target, forward_only=True)
        hp.close()
        hm.close()
        fd = (lp[0] - lm[0]) / (2 * eps)
        assert abs(grad[0, q] - fd) <= 1e-6 * max(abs(fd), np.abs(grad).max()), (q, grad[0, q], fd)
    h.close()
    ht.close()
