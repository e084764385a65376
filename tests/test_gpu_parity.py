"""Parity of the B200 path (through the C ABI) with the oracle and the reference's own GPU code.

Tolerances (FP64 everywhere):
  * states over the first 1000 RK4 steps: max|dS| <= 1e-10 (gate of the task);
    observed differences are rounding-level (~1e-14).
  * magnetisations per row: <= 1e-12 absolute; energy per site: <= 1e-12.
  * reference GPU integrator (oracle/_ref/libref_gpu.so): same tolerances.
"""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
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


def _pair(oracle, kind, dims, **kw):
    from classical_mcmc_spin_b200.lattice import Lattice
    if kind == "kitaev":
        lat = Lattice.kitaev(*dims, **kw)
        okw = {("direction" if k == "field_direction" else "g" if k == "g_factor" else k): v for k, v in kw.items()}
        o = oracle.OracleLattice.kitaev(*dims, **okw)
    else:
        lat = Lattice.pyrochlore_non_kramer(*dims, **kw)
        okw = {("direction" if k == "field_direction" else k): v for k, v in kw.items()}
        o = oracle.OracleLattice.pyrochlore_nk(*dims, **okw)
    return lat, o


def test_plain_rk4_1000_steps_matches_oracle(api, oracle):
    """Plain MD (Kitaev 24x24, 1152 spins, K=-1, G=0.25, G'=-0.02), 1000 RK4 steps, every step saved."""
    lat, o = _pair(oracle, "kitaev", (24, 24, 1))
    s0 = _spins(lat.lattice_size, 1)
    h = lat.to_gpu()
    api.set_gpu_spins(h, s0)
    traj, obs, times = api.integrate_gpu(h, 0.0, 9.995, 0.01, 1, "rk4", with_states=True)
    assert len(times) == 1001
    rows, fin = o.md_rk4(s0, 0.0, 9.995, 0.01, 1, gpu_loop=True)
    assert len(rows) == 1001
    np.testing.assert_array_equal(times, rows[:, 0])
    np.testing.assert_array_equal(traj[0][1], s0)
    assert np.abs(traj[-1][1] - fin).max() <= TOL_S
    assert np.abs(api.get_gpu_spins(h) - fin).max() <= TOL_S
    assert np.abs(obs[:, :9] - rows[:, 1:10]).max() <= TOL_M
    assert np.abs(obs[:, 9] - rows[:, 10]).max() <= TOL_M


def test_plain_rk4_matches_boost_form_oracle(api, oracle):
    """Same run against the oracle's odeint-style RK4 (the reference CPU integrator's arithmetic)."""
    lat, o = _pair(oracle, "kitaev", (24, 24, 1))
    s0 = _spins(lat.lattice_size, 2)
    h = lat.to_gpu()
    api.set_gpu_spins(h, s0)
    traj, obs, times = api.integrate_gpu(h, 0.0, 9.995, 0.01, 10, "rk4", with_states=True)
    # integrate_const stops at the last t0 + k dt <= T1 + eps, the GPU loop at
    # the first t >= T1: T1 = 10.005 gives the same 1000 steps.
    rows, fin = o.md_rk4(s0, 0.0, 10.005, 0.01, 10)
    assert len(rows) == len(obs) == 101
    np.testing.assert_allclose(times, rows[:, 0], rtol=0, atol=1e-12)
    assert np.abs(obs[:, :9] - rows[:, 1:10]).max() <= TOL_M
    assert np.abs(obs[:, 9] - rows[:, 10]).max() <= TOL_M
    assert np.abs(traj[-1][1] - fin).max() <= TOL_S


def test_driven_rk4_matches_oracle(api, oracle):
    lat, o = _pair(oracle, "kitaev", (6, 6, 1))
    s0 = _spins(lat.lattice_size, 3)
    fin1, fin2 = np.tile(R111, 2), np.tile([0.0, 1.0, 0.0], 2)
    fd = lat.rotate_pulse(fin1, fin2)
    h = lat.to_gpu()
    api.set_gpu_spins(h, s0)
    api.set_gpu_pulse(h, fd, 0.5, 0.5, 1.3, 0.3, 1.1)
    traj, obs, times = api.integrate_gpu(h, -0.5, 2.0, 0.01, 1, "rk4", with_states=False)
    o.set_pulse(fin1, 0.3, fin2, 1.1, 0.5, 0.5, 1.3)
    rows, fin = o.md_rk4(s0, -0.5, 2.0, 0.01, 1, gpu_loop=True)
    assert len(rows) == len(obs)
    assert np.abs(obs[:, :9] - rows[:, 1:10]).max() <= TOL_M
    assert np.abs(api.get_gpu_spins(h) - fin).max() <= TOL_S


def test_pyrochlore_with_field_matches_oracle(api, oracle):
    kw = dict(h=0.2, field_direction=R111, Jzz=1.0, Jpm=0.05, Jpmpm=0.02)
    lat, o = _pair(oracle, "pyro", (4, 4, 4), **kw)
    s0 = _spins(lat.lattice_size, 4)
    h = lat.to_gpu()
    assert h.layout_info()["bonds_per_site"] == 6
    api.set_gpu_spins(h, s0)
    traj, obs, times = api.integrate_gpu(h, 0.0, 4.9975, 0.005, 5, "rk4", with_states=False)
    rows, fin = o.md_rk4(s0, 0.0, 4.9975, 0.005, 5, gpu_loop=True)
    assert len(rows) == len(obs)
    assert np.abs(obs[:, :9] - rows[:, 1:10]).max() <= TOL_M
    assert np.abs(obs[:, 9] - rows[:, 10]).max() <= TOL_M
    assert np.abs(api.get_gpu_spins(h) - fin).max() <= TOL_S


def test_batch_pump_probe_matches_oracle(api, oracle):
    """Pump-only / probe-only / pump+probe trajectories of a delay scan in one launch."""
    from classical_mcmc_spin_b200.states import zigzag_honeycomb
    lat, o = _pair(oracle, "kitaev", (6, 6, 1))
    s0 = zigzag_honeycomb(6, 6, 1, tilt_sigma=0.05, seed=2).ravel()
    fin = np.tile(R111, 2)
    fd = lat.rotate_pulse(fin, fin)
    taus = [0.0, 0.7, 1.5]
    t1, t2, a1, a2 = [], [], [], []
    for tau in taus:
        for (x1, x2) in ((0.5, 0.0), (0.0, 0.5), (0.5, 0.5)):
            t1.append(0.0); t2.append(tau); a1.append(x1); a2.append(x2)
    h = lat.to_gpu()
    nsteps = 300
    obs, final = api.run_batch(h, s0, nsteps, 0.01, T0=-1.0, t1=t1, t2=t2, a1=a1, a2=a2, d1=fd[:6], d2=fd[6:],
                               width=0.5, freq=0.0, shared_initial=True)
    B = len(t1)
    states = np.tile(s0, (B, 1))
    st, oobs = o.batch_rk4(states, t1, t2, np.array(a1) / 0.5, np.array(a2) / 0.5, 0.5, 0.5, 0.0, fin, fin, -1.0,
                           0.01, nsteps)
    assert obs.shape == (B, nsteps + 1, 10)
    assert np.abs(obs[:, :, :9] - oobs[:, :, :9]).max() <= TOL_M
    assert np.abs(obs[:, :, 9] - oobs[:, :, 9]).max() <= TOL_M
    assert np.abs(final - st).max() <= TOL_S


def test_integrate_gpu_batched_matches_reference(api, oracle):
    """integrate_gpu_batched vs the reference's own implementation (oracle/_ref)."""
    if not oracle.ref_available("libref_gpu.so"):
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    lat, o = _pair(oracle, "kitaev", (4, 4, 1))
    s0 = _spins(lat.lattice_size, 13)
    fin = np.tile(R111, 2)
    fd = lat.rotate_pulse(fin, fin)
    tau2 = np.array([102.0, 0.0, 0.5, 1.0, 1.5])
    fr, afm = o.frames()
    ref = oracle.RefGPU(o.ell(), o.n_atoms)
    ref.set_pulse(fd, 0.5, 0.5, 0.0, 0.0, 0.0)
    rt, rm = ref.batched(s0, tau2, afm, fr, -1.0, 2.0, 0.01)
    ref.close()
    h = lat.to_gpu()
    api.set_gpu_pulse(h, fd, 0.5, 0.5, 0.0, 0.0, 0.0)
    res = api.integrate_gpu_batched(h, s0, tau2, afm, fr, -1.0, 2.0, 0.01)
    np.testing.assert_array_equal(res.times, rt)
    assert np.abs(res.mag_data.reshape(len(rt), len(tau2), 9) - rm).max() <= TOL_M


def test_plain_matches_reference_gpu_integrator(api, oracle):
    if not oracle.ref_available("libref_gpu.so"):
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    lat, o = _pair(oracle, "kitaev", (24, 24, 1))
    s0 = _spins(lat.lattice_size, 5)
    ref = oracle.RefGPU(o.ell(), o.n_atoms)
    ref.set_spins(s0)
    rt, rs = ref.integrate(0.0, 2.0, 0.01, save_interval=20, method="rk4")
    ref.close()
    h = lat.to_gpu()
    api.set_gpu_spins(h, s0)
    traj, obs, times = api.integrate_gpu(h, 0.0, 2.0, 0.01, 20, "rk4")
    np.testing.assert_array_equal(times, rt)
    assert np.abs(np.stack([s for _, s in traj]) - rs).max() <= 1e-12


@pytest.mark.parametrize("name", ["ref_gpu_rk4_kitaev.npz", "ref_gpu_rk4_kitaev24.npz"])
def test_plain_matches_golden(api, name):
    p = GOLDEN / name
    if not p.exists():
        pytest.skip("golden fixture not generated")
    g = np.load(p)
    from classical_mcmc_spin_b200.lattice import Lattice
    lat = Lattice.kitaev(int(g["d1"]), int(g["d2"]), 1)
    h = lat.to_gpu()
    api.set_gpu_spins(h, g["init"])
    T1 = float(g["T1"]) if "T1" in g else 2.0
    traj, obs, times = api.integrate_gpu(h, 0.0, T1, float(g["dt"]), int(g["save_interval"]), "rk4")
    np.testing.assert_array_equal(times, g["times"])
    assert np.abs(np.stack([s for _, s in traj]) - g["states"]).max() <= 1e-12


def test_energy_and_magnetization_api(api, oracle):
    lat, o = _pair(oracle, "kitaev", (6, 6, 1), h=0.3, field_direction=(0.1, 0.9, 0.2), Ka=0.1, Kc=-0.2)
    s0 = _spins(lat.lattice_size, 7)
    h = lat.to_gpu()
    api.set_gpu_spins(h, s0)
    assert abs(api.compute_energy_gpu(h) - o.energy(s0)) <= 1e-12 * lat.lattice_size
    ml, ms = api.compute_magnetization_gpu(h)
    S = s0.reshape(-1, 3)
    np.testing.assert_allclose(ml, S.mean(axis=0), atol=1e-15)
    sign = np.where(np.arange(len(S)) % 2 == 0, 1.0, -1.0)
    np.testing.assert_allclose(ms, (S * sign[:, None]).mean(axis=0), atol=1e-15)
    row = api.observables_gpu(h)
    np.testing.assert_allclose(row[:9], o.magnetizations(s0), atol=1e-15)


def test_step_and_normalize(api, oracle):
    lat, o = _pair(oracle, "kitaev", (4, 4, 1))
    s0 = _spins(lat.lattice_size, 8)
    h = lat.to_gpu()
    api.set_gpu_spins(h, s0)
    api.step_gpu(h, 0.0, 0.01, "rk4")
    assert np.abs(api.get_gpu_spins(h) - o.rk4_step(s0, 0.0, 0.01, gpu_form=True)).max() <= 1e-14
    api.set_gpu_spins(h, 2.0 * s0)
    api.normalize_spins_gpu(h, 1.0)
    np.testing.assert_allclose(api.get_gpu_spins(h), s0, atol=1e-15)


def test_errors_are_status_codes(api, native):
    from classical_mcmc_spin_b200.lattice import Lattice
    from classical_mcmc_spin_b200._native import CmdError
    lat = Lattice.kitaev(4, 4, 1)
    h = lat.to_gpu()
    with pytest.raises(CmdError) as e:
        api.step_gpu(h, 0.0, 0.01)
    assert e.value.code == native.CMD_ERR_STATE
    bad = _spins(lat.lattice_size, 1)
    bad[5] = np.nan
    with pytest.raises(CmdError) as e:
        api.set_gpu_spins(h, bad)
    assert e.value.code == native.CMD_ERR_NONFINITE
    api.set_gpu_spins(h, _spins(lat.lattice_size, 1))
    with pytest.raises(ValueError):
        api.step_gpu(h, 0.0, 0.01, "rk99")
    odd = Lattice.kitaev(4, 4, 1, J2_A=0.1, J2_B=0.1).to_gpu()    # 9 bonds/site: no kernel instance
    api.set_gpu_spins(odd, _spins(32, 1))
    with pytest.raises(CmdError) as e:
        api.step_gpu(odd, 0.0, 0.01)
    assert e.value.code == native.CMD_ERR_UNSUPPORTED


@pytest.mark.parametrize("kind", ["kitaev", "pyro"])
def test_every_kernel_variant_matches_oracle(api, oracle, kind):
    """Each resident-kernel variant that fits the lattice gives the oracle's trajectory."""
    if kind == "kitaev":
        lat, o = _pair(oracle, "kitaev", (24, 24, 1))
    else:
        lat, o = _pair(oracle, "pyro", (4, 4, 4), h=0.2, field_direction=R111, Jzz=1.0, Jpm=0.05, Jpmpm=0.02)
    s0 = _spins(lat.lattice_size, 21)
    fin = np.tile(R111, lat.N_atoms)
    fd = lat.rotate_pulse(fin, fin)
    o.set_pulse(fin, 0.1, fin, 0.6, 0.5, 0.5, 0.7)
    rows, ofin = o.md_rk4(s0, -0.5, 1.495, 0.01, 5, gpu_loop=True)
    h = lat.to_gpu()
    fits = [i for i, _, f in h.variants() if f]
    assert fits
    for v in fits:
        h.set_variant(v)
        assert h.get_variant() == v
        api.set_gpu_spins(h, s0)
        api.set_gpu_pulse(h, fd, 0.5, 0.5, 0.7, 0.1, 0.6)
        _, obs, times = api.integrate_gpu(h, -0.5, 1.495, 0.01, 5, "rk4", with_states=False)
        assert len(obs) == len(rows), v
        assert np.abs(obs[:, :9] - rows[:, 1:10]).max() <= TOL_M, v
        assert np.abs(obs[:, 9] - rows[:, 10]).max() <= TOL_M, v
        assert np.abs(api.get_gpu_spins(h) - ofin).max() <= TOL_S, v


def test_autotune_picks_a_fitting_variant(api, oracle):
    lat, o = _pair(oracle, "kitaev", (8, 8, 1))
    h = lat.to_gpu()
    api.set_gpu_spins(h, _spins(lat.lattice_size, 3))
    best, ms = h.autotune(16, 20)
    fits = {i for i, _, f in h.variants() if f}
    assert best in fits and ms[best] > 0
    assert all((ms[i] > 0) == (i in fits) for i in range(len(ms)))
    assert h.get_variant() == best


def test_cubic_pyrochlore_cell_matches_oracle(api, oracle):
    """16-site conventional cubic cells, grouped into the 4-site kernel classes."""
    kw = dict(h=0.2, field_direction=R111, Jzz=1.0, Jpm=0.05, Jpmpm=0.02, cubic=True)
    lat, o = _pair(oracle, "pyro", (2, 2, 2), **kw)
    s0 = _spins(lat.lattice_size, 22)
    fin16 = np.tile(R111, 16)
    fd = lat.rotate_pulse(fin16, fin16)
    h = lat.to_gpu()
    assert h.layout_info()["sites_per_group"] == 4
    api.set_gpu_spins(h, s0)
    api.set_gpu_pulse(h, fd, 0.4, 0.5, 0.0, 0.2, 0.7)
    _, obs, times = api.integrate_gpu(h, 0.0, 1.4975, 0.005, 5, "rk4", with_states=False)
    o.set_pulse(fin16, 0.2, fin16, 0.7, 0.4, 0.5, 0.0)
    rows, fin = o.md_rk4(s0, 0.0, 1.4975, 0.005, 5, gpu_loop=True)
    assert len(rows) == len(obs)
    assert np.abs(obs[:, :9] - rows[:, 1:10]).max() <= TOL_M
    assert np.abs(obs[:, 9] - rows[:, 10]).max() <= TOL_M
    assert np.abs(api.get_gpu_spins(h) - fin).max() <= TOL_S


def test_max_dsdt_no_drive_matches_oracle(api, native, oracle):
    """cmd_max_dsdt_no_drive (the 2DCS stationarity check) on random and stationary states, with a pulse set
    (which it must ignore)."""
    import ctypes as C
    for kind, dims, kw in (("kitaev", (6, 6, 1), dict(h=0.3, field_direction=(0.0, 1.0, 0.0))),
                           ("pyro", (2, 2, 2), dict(h=0.2, field_direction=R111, Jzz=1.0, Jpm=0.05, Jpmpm=0.02))):
        lat, o = _pair(oracle, kind, dims, **kw)
        h = lat.to_gpu()
        fin = np.tile(R111, lat.N_atoms)
        api.set_gpu_pulse(h, lat.rotate_pulse(fin, fin), 0.5, 0.5, 0.7, 0.0, 0.0)
        for s0 in (_spins(lat.lattice_size, 40), np.tile(np.asarray(kw["field_direction"]) /
                                                      np.linalg.norm(kw["field_direction"]), lat.lattice_size)):
            api.set_gpu_spins(h, s0)
            v = C.c_double()
            native.check(native.lib().cmd_max_dsdt_no_drive(h.ptr, C.byref(v)), "max_dsdt")
            ref = o.max_dsdt_no_drive(s0)
            assert abs(v.value - ref) <= 1e-13 * max(1.0, ref), (kind, v.value, ref)
