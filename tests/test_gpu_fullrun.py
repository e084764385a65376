"""Full-run gates.

From random spins the Kitaev and pyrochlore models are chaotic: two FP64 RK4 arithmetic orders
(the reference's own CPU and GPU steppers included) part at ~1e-6 by t ~ 50.  So full runs are
gated on properties that do not depend on the chaotic phase:
  * |S_i| drift and relative energy drift over the whole run within 2x of the oracle's;
  * |FFT(M)| over the coherent window (the first 2000 steps, where states agree to ~1e-12) within
    1e-6 relative of the oracle's, computed like the reference reader (mean-subtract, fft,
    fftshift, abs);
  * at the benchmark's full sizes: finite rows and unit norms to the RK4 drift level.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

R111 = np.ones(3) / np.sqrt(3.0)


@pytest.fixture(scope="module")
def api(native):
    from classical_mcmc_spin_b200 import gpu_api
    return gpu_api


def _spins(n, seed):
    from classical_mcmc_spin_b200.states import random_unit_spins
    return random_unit_spins(n, seed).ravel()


def _norm_dev(s):
    return np.abs(np.linalg.norm(np.asarray(s).reshape(-1, 3), axis=1) - 1.0)


def _drifts(e_rows, state):
    """(max norm deviation, mean norm deviation, relative energy drift)."""
    nd = _norm_dev(state)
    return nd.max(), nd.mean(), abs(e_rows[-1] - e_rows[0]) / abs(e_rows[0])


def _within_2x(gpu, ora):
    for g, o in zip(gpu, ora):
        assert g <= 2.0 * o + 1e-15, (gpu, ora)


def test_config1_full_run_drift_within_2x_of_oracle(api, oracle):
    """Kitaev 24x24 (1152 spins), seed 1, 10^4 RK4 steps (T = 100)."""
    from classical_mcmc_spin_b200.lattice import Lattice
    lat = Lattice.kitaev(24, 24, 1)
    o = oracle.OracleLattice.kitaev(24, 24, 1)
    s0 = _spins(lat.lattice_size, 1)
    h = lat.to_gpu()
    api.set_gpu_spins(h, s0)
    _, obs, _ = api.integrate_gpu(h, 0.0, 99.995, 0.01, 100, "rk4", with_states=False)
    rows, fin = o.md_rk4(s0, 0.0, 99.995, 0.01, 100, gpu_loop=True)
    assert len(rows) == len(obs) == 101
    _within_2x(_drifts(obs[:, 9], api.get_gpu_spins(h)), _drifts(rows[:, 10], fin))


def test_config1_spectrum_over_coherent_window(api, oracle):
    from classical_mcmc_spin_b200.lattice import Lattice
    lat = Lattice.kitaev(24, 24, 1)
    o = oracle.OracleLattice.kitaev(24, 24, 1)
    s0 = _spins(lat.lattice_size, 1)
    h = lat.to_gpu()
    api.set_gpu_spins(h, s0)
    _, obs, _ = api.integrate_gpu(h, 0.0, 19.995, 0.01, 1, "rk4", with_states=False)
    rows, _ = o.md_rk4(s0, 0.0, 19.995, 0.01, 1, gpu_loop=True)

    def spec(m):
        return np.abs(np.fft.fftshift(np.fft.fft(m - m.mean(axis=0), axis=0), axes=0))

    for cols_gpu, cols_ora in ((slice(0, 3), slice(1, 4)), (slice(3, 6), slice(4, 7))):   # M_af, M_local
        fg, fo = spec(obs[:, cols_gpu]), spec(rows[:, cols_ora])
        assert np.abs(fg - fo).max() <= 1e-6 * np.abs(fo).max()


@pytest.mark.parametrize("L,steps", [(4, 20000), (8, 4000)])
def test_pyrochlore_full_run_drift_within_2x_of_oracle(api, oracle, L, steps):
    """Non-Kramers pyrochlore with a [111] field, dt = 0.005: 4^3 cells (1024 spins, resident) over
    2x10^4 steps and 8^3 cells (8192 spins, streamed) over 4000 steps."""
    from classical_mcmc_spin_b200.lattice import Lattice
    kw = dict(h=0.2, Jzz=1.0, Jpm=0.05, Jpmpm=0.02)
    lat = Lattice.pyrochlore_non_kramer(L, L, L, field_direction=R111, cubic=True, **kw)
    o = oracle.OracleLattice.pyrochlore_nk(L, L, L, direction=R111, cubic=True, **kw)
    s0 = _spins(lat.lattice_size, 5)
    h = lat.to_gpu()
    api.set_gpu_spins(h, s0)
    T1 = (steps - 0.5) * 0.005
    _, obs, _ = api.integrate_gpu(h, 0.0, T1, 0.005, 1000, "rk4", with_states=False)
    rows, fin = o.md_rk4(s0, 0.0, T1, 0.005, 1000, gpu_loop=True)
    assert len(rows) == len(obs)
    _within_2x(_drifts(obs[:, 9], api.get_gpu_spins(h)), _drifts(rows[:, 10], fin))


def test_config2_full_size_scan_properties(api, oracle):
    """The full 2DCS scan (768 trajectories x 1152 spins x 2x10^4 steps, T_start = -5): finite rows,
    norm drift of every trajectory at the RK4 level, and for the first and last trajectory within 2x
    of the oracle's norm drift over the same full run."""
    from classical_mcmc_spin_b200.lattice import Lattice
    from classical_mcmc_spin_b200.states import zigzag_honeycomb
    lat = Lattice.kitaev(24, 24, 1)
    o = oracle.OracleLattice.kitaev(24, 24, 1)
    s0 = zigzag_honeycomb(24, 24, 1, tilt_sigma=0.05, seed=2).ravel()
    fd = lat.rotate_pulse(np.tile(R111, 2), np.tile(R111, 2))
    taus = 100.0 * np.arange(256) / 255.0
    t1, t2, a1, a2 = [], [], [], []
    for tau in taus:
        for (x1, x2) in ((0.5, 0.0), (0.0, 0.5), (0.5, 0.5)):
            t1.append(0.0); t2.append(tau); a1.append(x1); a2.append(x2)
    h = lat.to_gpu()
    S = 20000
    obs, final = api.run_batch(h, s0, S, 0.01, T0=-5.0, t1=t1, t2=t2, a1=a1, a2=a2, d1=fd[:6], d2=fd[6:],
                               width=0.5, freq=0.0, shared_initial=True, save_interval=100)
    B = len(t1)
    assert obs.shape == (B, S // 100 + 1, 10) and np.isfinite(obs).all()
    nd = np.array([_norm_dev(final[b]).max() for b in range(B)])
    assert nd.max() <= 1e-7
    pick = [0, B - 1]
    fin = np.tile(R111, 2)
    st, _ = o.batch_rk4(np.tile(s0, (2, 1)), [t1[b] for b in pick], [t2[b] for b in pick],
                        [a1[b] / 0.5 for b in pick], [a2[b] / 0.5 for b in pick], 0.5, 0.5, 0.0, fin, fin, -5.0,
                        0.01, S, with_obs=False)
    for k, b in enumerate(pick):
        g, r = _norm_dev(final[b]), _norm_dev(st[k])
        assert g.max() <= 2.0 * r.max() + 1e-15 and g.mean() <= 2.0 * r.mean() + 1e-15


def test_config5_full_size_properties(native):
    """65536-spin pyrochlore x 32 trajectories x 2x10^4 steps (dt = 0.005, no drive): finite rows,
    norms and energy conserved to the RK4 level."""
    import ctypes as C
    import torch
    from classical_mcmc_spin_b200 import _native as nat
    from classical_mcmc_spin_b200.lattice import Lattice
    from classical_mcmc_spin_b200.states import random_unit_spins
    lat = Lattice.pyrochlore_non_kramer(16, 16, 16, h=0.2, field_direction=R111, cubic=True, Jzz=1.0, Jpm=0.05,
                                        Jpmpm=0.02)
    N, B, S, save = lat.lattice_size, 32, 20000, 1000
    h = lat.to_gpu()
    states = np.stack([random_unit_spins(N, 5000 + b).ravel() for b in range(B)])
    d_states = torch.tensor(states, dtype=torch.float64, device="cuda")
    rows = int(nat.lib().cmd_batch_rows(S, save))
    d_obs = torch.empty((B, rows, 10), dtype=torch.float64, device="cuda")
    d_fin = torch.empty_like(d_states)
    desc = nat.BatchDesc()
    desc.B, desc.states, desc.method = B, d_states.data_ptr(), nat.CMD_RK4
    desc.width, desc.T0, desc.dt, desc.n_steps, desc.save_interval = 1.0, 0.0, 0.005, S, save
    desc.obs, desc.final_states = d_obs.data_ptr(), d_fin.data_ptr()
    st = torch.cuda.Stream()           # a stream of its own (handle 0 would mean the library's stream)
    torch.cuda.synchronize()           # inputs written on torch's stream are complete
    nat.check(nat.lib().cmd_run_batch_device(h.ptr, C.byref(desc), C.c_void_p(st.cuda_stream), None),
              "cmd_run_batch_device")
    torch.cuda.synchronize()
    obs = d_obs.cpu().numpy()
    fin = d_fin.cpu().numpy()
    assert np.isfinite(obs).all()
    assert _norm_dev(fin).max() <= 1e-7
    e = obs[:, :, 9]
    assert (np.abs(e[:, -1] - e[:, 0]) / np.abs(e[:, 0])).max() <= 1e-7
