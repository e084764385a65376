"""Controlled RK45, fixed-step Dormand-Prince, the global-memory RK4 and uneven batches on the GPU.

Tolerances: controlled steps follow the oracle's restatement of the CPU path's
Boost.Odeint controller, so accepted / rejected step counts must agree exactly.
The embedded error estimate cancels about eight digits (|x_err| ~ tol while the
stages are O(1)), so rounding-level differences between the GPU's and the
host's FMA patterns move each new step size at the 1e-9 relative level: accepted
times agree to 1e-7 absolute after hundreds of steps, row observables to 1e-7,
and the states at T_end (both controllers land on it exactly) to 1e-9.
Fixed-step Dormand-Prince is checked against the reference's own GPU "dopri5"
(oracle/_ref) at <= 1e-12.
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


def _kitaev(oracle, d1, d2):
    from classical_mcmc_spin_b200.lattice import Lattice
    return Lattice.kitaev(d1, d2, 1), oracle.OracleLattice.kitaev(d1, d2, 1)


def _pyro(oracle, L):
    from classical_mcmc_spin_b200.lattice import Lattice
    kw = dict(Jzz=1.0, Jpm=0.05, Jpmpm=0.02)
    return (Lattice.pyrochlore_non_kramer(L, L, L, h=0.2, field_direction=R111, **kw),
            oracle.OracleLattice.pyrochlore_nk(L, L, L, h=0.2, direction=R111, **kw))


@pytest.mark.parametrize("tol", [1e-8, 1e-10])
def test_rk45_single_matches_oracle_controller(api, oracle, tol):
    lat, o = _kitaev(oracle, 6, 6)
    s0 = _spins(lat.lattice_size, 31)
    h = lat.to_gpu()
    api.set_tolerances(h, tol, tol)
    api.set_gpu_spins(h, s0)
    _, obs, times = api.integrate_gpu(h, 0.0, 3.0, 0.01, 1, "rk45", with_states=False, max_rows=20000)
    rows, fin, stats = o.md_dopri5(s0, 0.0, 3.0, 0.01, tol, tol)
    assert len(times) == len(rows), (len(times), len(rows), stats)
    assert times[-1] == rows[-1, 0] == 3.0
    assert np.abs(times - rows[:, 0]).max() <= 1e-7
    assert np.abs(obs[:, :9] - rows[:, 1:10]).max() <= 1e-7
    assert np.abs(obs[:, 9] - rows[:, 10]).max() <= 1e-7
    assert np.abs(api.get_gpu_spins(h) - fin).max() <= 1e-9


def test_rk45_driven_pyrochlore_matches_oracle(api, oracle):
    lat, o = _pyro(oracle, 2)
    s0 = _spins(lat.lattice_size, 32)
    fin4 = np.tile(R111, 4)
    fd = lat.rotate_pulse(fin4, fin4)
    h = lat.to_gpu()
    api.set_tolerances(h, 1e-10, 1e-10)
    api.set_gpu_spins(h, s0)
    api.set_gpu_pulse(h, fd, 0.5, 0.5, 0.9, 0.3, 1.0)
    _, obs, times = api.integrate_gpu(h, -0.5, 2.0, 0.01, 1, "rk45", with_states=False, max_rows=20000)
    o.set_pulse(fin4, 0.3, fin4, 1.0, 0.5, 0.5, 0.9)
    rows, fin, stats = o.md_dopri5(s0, -0.5, 2.0, 0.01, 1e-10, 1e-10)
    assert len(times) == len(rows)
    assert np.abs(times - rows[:, 0]).max() <= 1e-7
    assert np.abs(obs[:, :9] - rows[:, 1:10]).max() <= 1e-7
    assert np.abs(api.get_gpu_spins(h) - fin).max() <= 1e-9


def test_dopri5_fixed_matches_reference_gpu(api, oracle):
    if not oracle.ref_available("libref_gpu.so"):
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    lat, o = _kitaev(oracle, 6, 6)
    s0 = _spins(lat.lattice_size, 33)
    ref = oracle.RefGPU(o.ell(), o.n_atoms)
    ref.set_spins(s0)
    rt, rs = ref.integrate(0.0, 1.0, 0.01, save_interval=10, method="dopri5")
    ref.close()
    h = lat.to_gpu()
    api.set_gpu_spins(h, s0)
    traj, obs, times = api.integrate_gpu(h, 0.0, 1.0, 0.01, 10, "dopri5")
    np.testing.assert_array_equal(times, rt)
    assert np.abs(np.stack([s for _, s in traj]) - rs).max() <= 1e-12
    for r in range(len(rt)):
        assert np.abs(obs[r, :9] - o.magnetizations(rs[r])).max() <= 1e-13


def test_cash_karp_fixed_matches_reference_gpu(api, oracle):
    """The reference GPU "rk5" (Cash-Karp tableau, fixed step; the md_integrator of its example configs)."""
    if not oracle.ref_available("libref_gpu.so"):
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    lat, o = _kitaev(oracle, 6, 6)
    s0 = _spins(lat.lattice_size, 35)
    ref = oracle.RefGPU(o.ell(), o.n_atoms)
    ref.set_spins(s0)
    rt, rs = ref.integrate(0.0, 1.0, 0.01, save_interval=10, method="rk5")
    ref.close()
    h = lat.to_gpu()
    api.set_gpu_spins(h, s0)
    traj, obs, times = api.integrate_gpu(h, 0.0, 1.0, 0.01, 10, "rk5")
    np.testing.assert_array_equal(times, rt)
    assert np.abs(np.stack([s for _, s in traj]) - rs).max() <= 1e-12
    for r in range(len(rt)):
        assert np.abs(obs[r, :9] - o.magnetizations(rs[r])).max() <= 1e-13
    api.set_gpu_spins(h, s0)                       # one step through cmd_step as well
    api.step_gpu(h, 0.0, 0.01, "rk5")
    ref = oracle.RefGPU(o.ell(), o.n_atoms)
    ref.set_spins(s0)
    ref.step(0.0, 0.01, method="rk5")
    assert np.abs(api.get_gpu_spins(h) - ref.get_spins()).max() <= 1e-14
    ref.close()


def test_streamed_rk4_for_large_lattice(api, oracle):
    """48x48 honeycomb (4608 spins) does not fit one CTA: RK4 runs on a 4-CTA cluster."""
    lat, o = _kitaev(oracle, 48, 48)
    s0 = _spins(lat.lattice_size, 34)
    h = lat.to_gpu()
    api.set_gpu_spins(h, s0)
    _, obs, times = api.integrate_gpu(h, 0.0, 0.995, 0.01, 10, "rk4", with_states=False)
    rows, fin = o.md_rk4(s0, 0.0, 0.995, 0.01, 10, gpu_loop=True)
    assert len(rows) == len(obs)
    assert np.abs(obs[:, :9] - rows[:, 1:10]).max() <= 1e-12
    assert np.abs(obs[:, 9] - rows[:, 10]).max() <= 1e-12
    assert np.abs(api.get_gpu_spins(h) - fin).max() <= 1e-10


def test_uneven_batch_rk45_matches_oracle(api, oracle):
    """Honeycomb L in {4, 6, 8} and pyrochlore L in {1, 2} in one persistent launch."""
    cases = []
    for L in (4, 6, 8, 6):
        lat, o = _kitaev(oracle, L, L)
        cases.append((lat, o))
    for L in (1, 2):
        cases.append(_pyro(oracle, L))
    handles = [c[0].to_gpu() for c in cases]
    specs = []
    for i, ((lat, o), h) in enumerate(zip(cases, handles)):
        specs.append(dict(handle=h, state=_spins(lat.lattice_size, 40 + i), T0=0.0, T1=1.5, dt=0.01,
                          max_rows=5000))
    out = api.run_uneven(specs, "rk45", 1e-10, 1e-10)
    for i, ((lat, o), sp) in enumerate(zip(cases, specs)):
        rows, fin, stats = out[i]
        orows, ofin, ostats = o.md_dopri5(sp["state"], 0.0, 1.5, 0.01, 1e-10, 1e-10)
        assert stats[3] == 0 and stats[1] == ostats[0] and stats[2] == ostats[1], (i, stats, ostats)
        assert len(rows) == len(orows)
        assert np.abs(rows[:, 0] - orows[:, 0]).max() <= 1e-7
        assert np.abs(rows[:, 1:] - orows[:, 1:]).max() <= 1e-7
        assert np.abs(fin - ofin).max() <= 1e-9


def test_uneven_batch_rk4_max_steps_and_errors(api, oracle):
    from classical_mcmc_spin_b200._native import CmdError
    lat, o = _kitaev(oracle, 4, 4)
    h = lat.to_gpu()
    s0 = _spins(lat.lattice_size, 50)
    out = api.run_uneven([dict(handle=h, state=s0, T0=0.0, T1=0.5, dt=0.01, max_rows=200)], "rk4")
    rows, fin, stats = out[0]
    orows, ofin = o.md_rk4(s0, 0.0, 0.5, 0.01, 1, gpu_loop=True)
    assert len(rows) == len(orows) and np.abs(fin - ofin).max() <= 1e-12
    out = api.run_uneven([dict(handle=h, state=s0, T0=0.0, T1=100.0, dt=0.01, max_rows=60)], "rk45", 1e-10,
                         1e-10, max_steps=50)
    assert out[0][2][1] == 50 and len(out[0][0]) == 51
    with pytest.raises(CmdError):
        api.run_uneven([dict(handle=h, state=s0, T0=0.0, T1=1.0, dt=0.01, max_rows=5)], "rk4")


def _rk45_case(oracle, kind, L):
    from classical_mcmc_spin_b200.lattice import Lattice
    if kind == "kitaev":
        return Lattice.kitaev(L, L, 1), oracle.OracleLattice.kitaev(L, L, 1)
    kw = dict(Jzz=1.0, Jpm=0.05, Jpmpm=0.02)
    return (Lattice.pyrochlore_non_kramer(L, L, L, h=0.2, field_direction=R111, cubic=True, **kw),
            oracle.OracleLattice.pyrochlore_nk(L, L, L, h=0.2, direction=R111, cubic=True, **kw))


@pytest.mark.parametrize("kind,L,driven", [("kitaev", 8, False), ("kitaev", 8, True), ("kitaev", 32, False),
                                           ("pyro", 4, True), ("pyro", 6, False), ("pyro", 8, False)])
def test_rk45_every_tiling_matches_oracle_controller(api, oracle, kind, L, driven):
    """Every on-chip tiling that holds the lattice (one CTA, 2- to 16-CTA clusters; 512 or 1024 threads) and
    the global-memory kernel: identical accepted / rejected counts, rows <= 1e-7, final state <= 1e-9."""
    lat, o = _rk45_case(oracle, kind, L)
    s0 = _spins(lat.lattice_size, 400 + L)
    h = lat.to_gpu()
    api.set_tolerances(h, 1e-10, 1e-10)
    T1 = 1.0
    if driven:
        fin = np.tile(R111, lat.N_atoms)
        api.set_gpu_pulse(h, lat.rotate_pulse(fin, fin), 0.6, 0.15, 1.3, 0.3, 0.55)
        o.set_pulse(fin, 0.3, fin, 0.55, 0.6, 0.15, 1.3)
    orows, ofin, ostats = o.md_dopri5(s0, 0.0, T1, 0.01, 1e-10, 1e-10)
    tilings = [(i, n) for i, n, fits in h.rk45_variants() if fits]
    assert tilings, "no on-chip tiling holds the lattice"
    for idx, name in tilings + [(-2, "global-memory kernel")]:
        h.set_rk45_variant(idx)
        assert h.get_rk45_variant() == idx
        api.set_gpu_spins(h, s0)
        _, obs, times = api.integrate_gpu(h, 0.0, T1, 0.01, 1, "rk45", with_states=False, max_rows=20000)
        assert len(times) == len(orows), (name, len(times), len(orows), ostats)
        assert times[-1] == T1, name
        assert np.abs(times - orows[:, 0]).max() <= 1e-7, name
        assert np.abs(obs[:, :9] - orows[:, 1:10]).max() <= 1e-7, name
        assert np.abs(obs[:, 9] - orows[:, 10]).max() <= 1e-7, name
        assert np.abs(api.get_gpu_spins(h) - ofin).max() <= 1e-9, name
    h.close()


def test_rk45_tiling_autotuner_pins_a_fitting_tiling(api, oracle):
    lat, o = _rk45_case(oracle, "kitaev", 32)
    s0 = _spins(lat.lattice_size, 77)
    h = lat.to_gpu()
    api.set_tolerances(h, 1e-10, 1e-10)
    api.set_gpu_spins(h, s0)
    best, ms = h.autotune_rk45(4, 20)
    fits = {i for i, _, f in h.rk45_variants() if f}
    assert best in fits and h.get_rk45_variant() == best
    assert all((ms[i] > 0) == (i in fits) for i in range(len(ms)))
    api.set_gpu_spins(h, s0)
    _, obs, times = api.integrate_gpu(h, 0.0, 0.5, 0.01, 1, "rk45", with_states=False, max_rows=20000)
    orows, ofin, _ = o.md_dopri5(s0, 0.0, 0.5, 0.01, 1e-10, 1e-10)
    assert len(times) == len(orows) and np.abs(obs[:, :9] - orows[:, 1:10]).max() <= 1e-7
    h.close()


def test_rk45_saved_states_on_chip(api, oracle):
    """States of every accepted step (the trajectory output of integrate_gpu) from the on-chip kernel."""
    lat, o = _rk45_case(oracle, "kitaev", 6)
    s0 = _spins(lat.lattice_size, 78)
    h = lat.to_gpu()
    api.set_tolerances(h, 1e-8, 1e-8)
    api.set_gpu_spins(h, s0)
    assert h.get_rk45_variant() >= 0
    traj, obs, times = api.integrate_gpu(h, 0.0, 0.6, 0.01, 1, "rk45", with_states=True, max_rows=20000)
    h.set_rk45_variant(-2)
    api.set_gpu_spins(h, s0)
    traj2, obs2, times2 = api.integrate_gpu(h, 0.0, 0.6, 0.01, 1, "rk45", with_states=True, max_rows=20000)
    assert len(traj) == len(traj2) == len(times)
    np.testing.assert_array_equal(traj[0][1], s0)
    assert max(np.abs(a[1] - b[1]).max() for a, b in zip(traj, traj2)) <= 1e-10
    h.close()
